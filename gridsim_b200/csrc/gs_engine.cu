// gs_engine.cu — the batched Newton-Raphson load-flow engine and its C ABI (sm_100a).
//
// One Newton iteration of a batch of B systems (contingencies, load scalings, requests) of one grid:
//   1. k_mismatch_jac  — per (bus, system): injections P_i, Q_i over row i of Y (FP64, the outaged
//                        branch's four cells replaced by their reduced values), mismatch into the
//                        right-hand side, max-norm per system, Jacobian blocks H/N/M/L written straight
//                        into the LU slots of the shared static-pivot pattern
//                        (ComputeInjections :269-289, mismatch :216-235, RefillJacobian :342-380 of
//                        src/GridSim.Core/PowerFlow/SparseNewtonRaphsonPowerFlow.cs);
//   2. k_status        — per system: converged / diverged / cap / non-finite tests in the reference's
//                        order (RunNewton :235-238, NewtonShell.DivergedBeyondLimit :177-178);
//   3. factorisation   — per elimination-tree level, two phases (pivots, upper and forward entries; then
//                        lower entries): every entry its own sparse dot product over the row subtree of its
//                        node (k_level launches for the wide levels, one k_persistent launch for the
//                        narrow top of the tree);
//   4. backward substitution, levels top down (k_persistent, then k_level launches);
//   5. k_dxmax, k_update — max |dx| per system, damped update with the Vm floor
//                        (NewtonShell.ApplyStep :128-136, MaxUndampedStep 0.4, VmFloorPu 0.01).
// Steps 3-5 are captured once per batch into a CUDA graph and replayed every iteration; the host reads
// one counter (systems still active) per iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "gs_host.h"
#include "gs_kernels.cuh"

namespace gs {

constexpr double kMaxUndampedStep = 0.4;
constexpr double kRefineBelowPu = 1e-3;
constexpr double kVmFloorPu = 0.01;

__device__ __forceinline__ void atomicMaxNonNeg(unsigned long long* a, double v) {
    atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// The system of batch position `idx`: the position itself, or (few-systems path) the idx-th listed system;
// -1 past the end of the list.
__device__ __forceinline__ int sysAt(int idx, const int* list, int nList) {
    if (!list) return idx;
    return idx < nList ? list[idx] : -1;
}

// The voltage-dependent (ZIP) load of bus i at vm (ZipLoad, Model/Model.cs:45-63; NewtonShell.ZipDeviationPu :396-402,
// ZipJacobianDiagPu :407-413): its deviation from the nominal load pd, qd (pu) and the deviation's derivative in vm.
// False for a constant-power bus.
__device__ __forceinline__ bool zipLoad(const DevGrid& g, int i, double vm, double pd, double qd, double& dP, double& dQ,
                                        double& dPdV, double& dQdV) {
    if (!g.zip) return false;
    const double* c = g.zip + 6 * (size_t)i;
    const double ap = c[0], bp = c[1], cp = c[2], aq = c[3], bq = c[4], cq = c[5];
    if (ap == 0.0 && bp == 0.0 && aq == 0.0 && bq == 0.0) return false;
    dP = pd * (ap * vm * vm + bp * vm + cp - 1.0);
    dQ = qd * (aq * vm * vm + bq * vm + cq - 1.0);
    dPdV = pd * (2.0 * ap * vm + bp);
    dQdV = qd * (2.0 * aq * vm + bq);
    return true;
}

// ---------------------------------------------------------------------------------------------
// 1. mismatch + Jacobian fill of bus i of system s: injections over row i of Y (the outaged branch's four cells
//    replaced by their reduced values), the mismatch into the right-hand side (and its FP64 copy in mixed
//    precision), the Jacobian blocks of row i into their LU slots; folds |mismatch| into localMax and sets bad
//    (1: mismatch not finite, 2: Jacobian not finite).
template <typename T>
__device__ __forceinline__ void busMismatchJac(const DevGrid& g, const DevBatch& b, int i, int s, int fillJac, double* pOut,
                                               double* qOut, double& localMax, int& bad) {
    const size_t B = (size_t)b.B;
    const double vmi = b.vm[i * B + s], vai = b.va[i * B + s];
    // Grids analysed with every bus's P and Q rows (qlim): the bus's type in this system (3 reference, 2 PV, 1 PQ,
    // 0 removed) decides which rows are equations. A reference or removed bus keeps identity P and Q rows, a PV bus
    // an identity Q row (their steps are 0, their mismatches are not equations); a bus that starts PV or reference
    // and is PQ now (switched at a Q limit, or left without units) holds Q at qspecSys.
    const int gt = g.busType[i];
    const int et = g.qlim ? b.effType[i * B + s] : gt;
    const bool pId = g.qlim && (et == 3 || et == 0);
    const bool qId = g.qlim && et != 1;
    const int kp = g.busP[i], kq = g.busQ[i];
    const bool fill = fillJac && (kp >= 0 || kq >= 0);
    T* lu = (T*)b.lu;
    // one pass over row i: the injections, and the off-diagonal Jacobian blocks from the same sin/cos (they do not
    // need P, Q); the diagonal blocks follow from the sums
    double pi = 0.0, qi = 0.0, Gd = 0.0, Bd = 0.0;
    int pd = -1;
    const int p0 = g.yRowPtr[i], p1 = g.yRowPtr[i + 1];
    CellOverride ovr(g, b.outage[s], p0);
    for (int p = p0; p < p1; p++) {
        const int j = g.yCol[p];
        double G = g.yG[p], Bv = g.yB[p];
        ovr.at(g, p, G, Bv);
        double sn, cs;
        sincos(vai - b.va[j * B + s], &sn, &cs);
        const double vmj = b.vm[j * B + s];
        pi += vmj * (G * cs + Bv * sn);
        qi += vmj * (G * sn - Bv * cs);
        if (j == i) { pd = p; Gd = G; Bd = Bv; continue; }
        if (!fill) continue;
        const double H = pId ? 0.0 : vmi * vmj * (G * sn - Bv * cs);
        const double N = pId ? 0.0 : vmi * (G * cs + Bv * sn);
        const double M = qId ? 0.0 : -vmi * vmj * (G * cs + Bv * sn);
        const double L = qId ? 0.0 : vmi * (G * sn - Bv * cs);
        const int4 sl = *reinterpret_cast<const int4*>(g.ySlot + 4 * p);
        if (sl.x >= 0) lu[sl.x * B + s] = (T)H;
        if (sl.y >= 0) lu[sl.y * B + s] = (T)N;
        if (sl.z >= 0) lu[sl.z * B + s] = (T)M;
        if (sl.w >= 0) lu[sl.w * B + s] = (T)L;
        bad |= (isfinite(H) && isfinite(N) && isfinite(M) && isfinite(L)) ? 0 : 2;
    }
    const double P = vmi * pi, Q = vmi * qi;
    const double sc = b.loadScale ? b.loadScale[i * B + s] : 1.0;
    // a ZIP load's deviation comes off the mismatch, its derivative onto the N and L diagonals of a bus with a voltage
    // column (SparseNewtonRaphsonPowerFlow.cs:223-231, :241-248)
    double zdP = 0.0, zdQ = 0.0, zdPdV = 0.0, zdQdV = 0.0;
    const bool zip = zipLoad(g, i, vmi, sc * g.pload[i], sc * g.qload[i], zdP, zdQ, zdPdV, zdQdV);
    const bool vcol = zip && kq >= 0 && !qId;
    if (fill && pd >= 0) {
        const double H = pId ? 1.0 : -Q - Bd * vmi * vmi;
        const double N = pId ? 0.0 : P / vmi + Gd * vmi + (vcol ? zdPdV : 0.0);
        const double M = qId ? 0.0 : P - Gd * vmi * vmi;
        const double L = qId ? 1.0 : Q / vmi - Bd * vmi + (vcol ? zdQdV : 0.0);
        const int4 sl = *reinterpret_cast<const int4*>(g.ySlot + 4 * pd);
        if (sl.x >= 0) lu[sl.x * B + s] = (T)H;
        if (sl.y >= 0) lu[sl.y * B + s] = (T)N;
        if (sl.z >= 0) lu[sl.z * B + s] = (T)M;
        if (sl.w >= 0) lu[sl.w * B + s] = (T)L;
        bad |= (isfinite(H) && isfinite(N) && isfinite(M) && isfinite(L)) ? 0 : 2;
    }
    if (pOut) { pOut[i * B + s] = P; qOut[i * B + s] = Q; }
    double pspec = b.loadScale ? g.pgen[i] - sc * g.pload[i] : g.pgen[i] - g.pload[i];
    double qspec = b.loadScale ? g.qgen[i] - sc * g.qload[i] : g.qgen[i] - g.qload[i];
    if (b.specBus && b.specBus[s] == i) {  // a generator outage: the bus loses the unit's output
        pspec = (g.pgen[i] - b.specDp[s]) - sc * g.pload[i];
        qspec = (g.qgen[i] - b.specDq[s]) - sc * g.qload[i];
    }
    if (g.qlim) {
        if (gt == 2) b.qinj[i * B + s] = Q;
        if (et == 1 && gt != 1) qspec = b.qspecSys[i * B + s];
    }
    T* y = (T*)b.y;
    if (kp >= 0 && pId) {
        y[kp * B + s] = T(0);
        if (b.rhs64) b.rhs64[kp * B + s] = 0.0;
    } else if (kp >= 0) {
        const double f = pspec - P - zdP;
        y[kp * B + s] = (T)f;
        if (b.rhs64) b.rhs64[kp * B + s] = f;
        localMax = fmax(localMax, fabs(f));
        bad |= isfinite(f) ? 0 : 1;
    }
    if (kq >= 0 && qId) {
        y[kq * B + s] = T(0);
        if (b.rhs64) b.rhs64[kq * B + s] = 0.0;
    } else if (kq >= 0) {
        const double f = qspec - Q - zdQ;
        y[kq * B + s] = (T)f;
        if (b.rhs64) b.rhs64[kq * B + s] = f;
        localMax = fmax(localMax, fabs(f));
        bad |= isfinite(f) ? 0 : 1;
    }
}

// The batched kernel. Block (32, 8): lane = system, y = bus within the block.
template <typename T>
__global__ void __launch_bounds__(256) k_mismatch_jac(DevGrid g, DevBatch b, int fillJac, double* pOut, double* qOut,
                                                      const int* list, int nList) {
    const int lane = threadIdx.x, w = threadIdx.y;
    const int s = sysAt(blockIdx.y * 32 + lane, list, nList);
    const int i = blockIdx.x * 8 + w;
    double localMax = 0.0;
    int bad = 0;  // 1: mismatch not finite, 2: Jacobian not finite
    const bool live = i < g.n && s >= 0 && s < b.count && b.active[s];
    if (live) {
        busMismatchJac<T>(g, b, i, s, fillJac, pOut, qOut, localMax, bad);
    }
    __shared__ double red[8][32];
    __shared__ int redBad[8][32];
    red[w][lane] = localMax;
    redBad[w][lane] = bad;
    __syncthreads();
    if (w == 0 && s >= 0 && s < b.count) {
        double mx = red[0][lane];
        int anyBad = redBad[0][lane];
        for (int q = 1; q < 8; q++) { mx = fmax(mx, red[q][lane]); anyBad |= redBad[q][lane]; }
        if (mx > 0.0) atomicMaxNonNeg(&b.maxMis[s], mx);
        if (anyBad & 1) atomicOr(&b.flags[s], kFlagNonFinite);
        if (anyBad & 2) atomicOr(&b.flags[s], kFlagJacBad);
    }
}

// ---------------------------------------------------------------------------------------------
// 2. per-system Newton control (RunNewton :218-238): the tests in the reference's order. `iter` is the
//    system's step count so far. Returns whether the system takes another step; `activeCount[0]` counts
//    those, `activeCount[1]` those of them that refine their step (mixed precision).
__device__ __forceinline__ bool statusStep(const DevBatch& b, int s, int iter, double tol, double divLimit, int maxIter) {
    const double mis = __longlong_as_double((long long)b.maxMis[s]);
    b.maxMis[s] = 0ull;
    b.maxDx[s] = 0ull;
    const int fl = b.flags[s];
    if (fl & kFlagNonFinite) {  // a NaN mismatch never converges; the non-finite step then stops the run
        b.finalMis[s] = NAN;
        b.status[s] = GS_PF_NON_FINITE;
        b.active[s] = 0;
        return false;
    }
    if (fl & kFlagStepBad) {  // the previous step was refused: the run stops, state unchanged
        b.status[s] = GS_PF_MAX_ITERATIONS;
        b.active[s] = 0;
        return false;
    }
    b.finalMis[s] = mis;
    if (iter == 0) b.startMis[s] = mis;
    if (mis < tol) {
        b.status[s] = GS_PF_CONVERGED;
        b.convIters[s] = b.iters[s];
        b.active[s] = 0;
        return false;
    }
    if (mis > fmax(divLimit, b.startMis[s])) { b.status[s] = GS_PF_DIVERGED; b.active[s] = 0; return false; }
    if (iter >= maxIter) { b.status[s] = GS_PF_MAX_ITERATIONS; b.active[s] = 0; return false; }
    if (fl & kFlagJacBad) { b.status[s] = GS_PF_MAX_ITERATIONS; b.active[s] = 0; return false; }  // SolveStep refuses it
    // Mixed precision refines the FP32 step with the FP64 residual once the mismatch is small: far from the
    // root the Newton step is self-correcting and an FP32 step error of ~kappa * 2^-24 changes nothing.
    if (b.refine) {
        const int r = mis < kRefineBelowPu ? 1 : 0;
        b.refine[s] = r;
        if (r) atomicAdd(b.activeCount + 1, 1);
    }
    if (b.beforeLast) b.beforeLast[s] = mis;
    atomicAdd(b.activeCount, 1);
    return true;
}

// A batch in lock step: every active system has taken `iter` steps.
__global__ void k_status(DevBatch b, int iter, double tol, double divLimit, int maxIter) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.count || !b.active[s]) return;
    statusStep(b, s, iter, tol, divLimit, maxIter);
}

// ---- Q-limit enforcement (SparseNewtonRaphsonPowerFlow.Solve's Q-limit passes, SparseNewtonRaphsonPowerFlow.cs:118-160;
//      NewtonShell.ApplyQLimits :519-558, RevertBrokenPins :593-603, TryRevertPin :563-576). Every pass is a Newton run
//      of its own (its first mismatch is the divergence reference, the iteration cap counts its steps). When a pass
//      converges, PV buses whose generator Q is beyond the aggregate limits (by more than 1e-3 MVAr) become PQ with
//      Q held at the limit; if none does, pinned buses whose voltage crossed the set point (by 1e-4 pu) revert to
//      PV once each. Any change starts the next pass from the present state (up to 100 passes, then one last run
//      whose end is not a convergence); no change ends the solve converged.
constexpr double kQLimitTolMva = 1e-3;      // NewtonShell.cs:26
constexpr double kRevertVoltTolPu = 1e-4;   // NewtonShell.cs:31
constexpr int kMaxQPasses = 100;            // PowerFlowOptions.MaxQLimitPasses default (:101)
enum : int32_t { kQReverted = 16 };

__global__ void k_status_q(DevBatch b, double tol, double divLimit, int maxIter) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.count || !b.active[s]) return;
    b.qState[s] &= ~kQSkipStep;
    const int iter = b.passIter[s];
    const double mis = __longlong_as_double((long long)b.maxMis[s]);
    b.maxMis[s] = 0ull;
    b.maxDx[s] = 0ull;
    const int fl = b.flags[s];
    if (fl & kFlagNonFinite) { b.finalMis[s] = NAN; b.status[s] = GS_PF_NON_FINITE; b.active[s] = 0; return; }
    if (fl & kFlagStepBad) { b.status[s] = GS_PF_MAX_ITERATIONS; b.active[s] = 0; return; }
    b.finalMis[s] = mis;
    if (iter == 0) b.startMis[s] = mis;
    if (mis < tol) {
        if (b.qState[s] & kQFinalPass) {  // the last run converged, but the pass cap ends the solve unconverged
            b.status[s] = GS_PF_MAX_ITERATIONS;
            b.qState[s] |= kQFinalConverged;
            b.active[s] = 0;
            return;
        }
        b.qState[s] |= kQPending;  // the Q limits decide (k_qapply, k_qrevert, k_qfinish)
        return;
    }
    if (mis > fmax(divLimit, b.startMis[s])) { b.status[s] = GS_PF_DIVERGED; b.active[s] = 0; return; }
    if (iter >= maxIter) { b.status[s] = GS_PF_MAX_ITERATIONS; b.active[s] = 0; return; }
    if (fl & kFlagJacBad) { b.status[s] = GS_PF_MAX_ITERATIONS; b.active[s] = 0; return; }
    if (b.refine) {
        const int r = mis < kRefineBelowPu ? 1 : 0;
        b.refine[s] = r;
        if (r) atomicAdd(b.activeCount + 1, 1);
    }
    if (b.beforeLast) b.beforeLast[s] = mis;
    atomicAdd(b.activeCount, 1);
}

// TryRevertPin (NewtonShell.cs:563-576): a bus pinned at a limit whose voltage crossed its set point (by 1e-4 pu, on
// the side the limit pushes it) goes back to PV at the set point, once per solve.
__device__ __forceinline__ bool tryRevertPin(const DevGrid& g, const DevBatch& b, int i, int s, size_t idx) {
    const int pin = b.pinned[idx];
    if (b.effType[idx] != 1 || (pin != 1 && pin != -1) || b.reverted[idx] >= 1) return false;
    double vg = g.vm0[i];  // the set point (of the units left, after a generator outage)
    if (b.ovBus && b.ovBus[2 * s] == i && !isnan(b.ovVm[2 * s])) vg = b.ovVm[2 * s];
    else if (b.ovBus && b.ovBus[2 * s + 1] == i && !isnan(b.ovVm[2 * s + 1])) vg = b.ovVm[2 * s + 1];
    const double vm = b.vm[idx];
    if (!((pin == 1 && vm > vg + kRevertVoltTolPu) || (pin == -1 && vm < vg - kRevertVoltTolPu))) return false;
    b.effType[idx] = 2;
    b.vm[idx] = vg;
    b.pinned[idx] = 0;
    b.reverted[idx] += 1;
    return true;
}

// ApplyQLimits on the systems whose pass converged: grid (ceil(n / 8), B / 32), block (32, 8).
__global__ void k_qapply(DevGrid g, DevBatch b) {
    const int s = blockIdx.y * 32 + threadIdx.x, i = blockIdx.x * 8 + threadIdx.y;
    if (!g.qlimOn || i >= g.n || s >= b.count || !b.active[s] || !(b.qState[s] & kQPending) || g.busType[i] != 2) return;
    const size_t idx = (size_t)i * b.B + s;
    if (b.effType[idx] != 2) {  // with RevertQLimits a pinned bus may go back to PV in the same pass (:551-556)
        if (g.qlimRevert && tryRevertPin(g, b, i, s, idx)) atomicOr(&b.qState[s], kQChanged);
        return;
    }
    const double qd = (b.loadScale ? b.loadScale[idx] : 1.0) * g.qload[i];  // the bus's nominal load, pu
    // the generators' output: the injection plus the load drawn at the solved voltage (NewtonShell.cs:533-537)
    double zdP, zdQ = 0.0, zdPdV, zdQdV;
    zipLoad(g, i, b.vm[idx], 0.0, qd, zdP, zdQ, zdPdV, zdQdV);
    const double qGen = (b.qinj[idx] + qd + zdQ) * g.baseMva;
    // the aggregate limits of the bus's units (those left after a generator outage)
    const bool spec = b.specBus && b.specBus[s] == i;
    const double qmin = spec ? b.specQmin[s] : g.qminMvar[i], qmax = spec ? b.specQmax[s] : g.qmaxMvar[i];
    const bool fixed = qmin == qmax;
    if (qGen > qmax + kQLimitTolMva) {
        b.effType[idx] = 1;
        b.qspecSys[idx] = (spec ? qmax / g.baseMva : g.qmaxPu[i]) - qd;
        b.pinned[idx] = fixed ? 2 : 1;
        atomicOr(&b.qState[s], kQChanged);
    } else if (qGen < qmin - kQLimitTolMva) {
        b.effType[idx] = 1;
        b.qspecSys[idx] = (spec ? qmin / g.baseMva : g.qminPu[i]) - qd;
        b.pinned[idx] = fixed ? 2 : -1;
        atomicOr(&b.qState[s], kQChanged);
    }
}

// RevertBrokenPins on the systems whose pass converged without a switch.
__global__ void k_qrevert(DevGrid g, DevBatch b) {
    const int s = blockIdx.y * 32 + threadIdx.x, i = blockIdx.x * 8 + threadIdx.y;
    if (i >= g.n || s >= b.count || !b.active[s] || g.busType[i] != 2) return;
    const int st = b.qState[s];
    if (!(st & kQPending) || (st & kQChanged)) return;
    const size_t idx = (size_t)i * b.B + s;
    if (tryRevertPin(g, b, i, s, idx)) atomicOr(&b.qState[s], kQReverted);
}

// The end of a converged pass: a switch starts the next pass (this iteration's step is not taken), else converged.
__global__ void k_qfinish(DevBatch b, int maxPasses) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.count || !b.active[s]) return;
    const int st = b.qState[s];
    if (!(st & kQPending)) return;
    if (st & (kQChanged | kQReverted)) {
        b.qPass[s] += 1;
        b.passIter[s] = 0;
        b.qState[s] = kQSkipStep | (b.qPass[s] >= maxPasses ? kQFinalPass : 0);
        atomicAdd(b.activeCount, 1);
    } else {
        b.status[s] = GS_PF_CONVERGED;
        b.convIters[s] = b.iters[s];
        b.active[s] = 0;
        b.qState[s] = 0;
    }
}

// Systems admitted at different times (the request loop): each at its own step count. Systems that stop
// here are listed in done[1 ..], done[0] their number.
__global__ void k_status_each(DevBatch b, double tol, double divLimit, int maxIter, int* done) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.count || !b.active[s]) return;
    if (!statusStep(b, s, b.iters[s], tol, divLimit, maxIter)) done[1 + atomicAdd(done, 1)] = s;
}

// ---------------------------------------------------------------------------------------------
// 3. fused factorisation + forward substitution of one elimination-tree level.
//
// Warp layout of the LU kernels: S systems x P = 32 / S pair lanes (S = 8 for FP32, 4 for FP64, so that the
// lanes of one pair lane read exactly one 32-byte sector). An entry's index pairs are dealt round-robin to the
// P pair lanes; each lane accumulates its products, then a fixed butterfly over the pair lanes sums them (a
// fixed order: the result is deterministic). A warp therefore finishes a 32-pair batch in one round of loads
// instead of 32 / 8 rounds, and there are P times more warps per level than with one system per lane.
template <typename T>
struct Lay {
    static constexpr int S = sizeof(T) == 4 ? 8 : 4;  // systems per warp
    static constexpr int P = 32 / S;                  // pair lanes
};

// sum over pairs q in [q0, q1) of lu[a] * rhs[c] for this lane's system, complete in every pair lane.
template <typename T>
__device__ __forceinline__ T dotSP(const T* __restrict__ lu, const T* __restrict__ rhs, const int2* __restrict__ pr,
                                   int64_t q0, int64_t q1, size_t B, int s) {
    constexpr int S = Lay<T>::S, P = Lay<T>::P;
    const int lane = threadIdx.x & 31;
    const int pl = lane / S;
    T acc = T(0);
    // the next batch's index pairs are loaded while this batch's operands are in flight
    int2 next = q0 + lane < q1 ? __ldg(pr + q0 + lane) : make_int2(0, 0);
    for (int64_t base = q0; base < q1; base += 32) {
        const int cnt = (int)min((int64_t)32, q1 - base);
        const int2 mine = next;
        if (base + 32 < q1) next = base + 32 + lane < q1 ? __ldg(pr + base + 32 + lane) : make_int2(0, 0);
        T l[S], r[S];
#pragma unroll
        for (int u = 0; u < S; u++) {
            const int src = pl + P * u;
            const int a = __shfl_sync(0xffffffffu, mine.x, src);
            const int c = __shfl_sync(0xffffffffu, mine.y, src);
            const bool ok = src < cnt;
            l[u] = ok ? lu[a * B + s] : T(0);
            r[u] = ok ? rhs[c * B + s] : T(0);
        }
#pragma unroll
        for (int u = 0; u < S; u++) acc += l[u] * r[u];
    }
#pragma unroll
    for (int off = S; off < 32; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    return acc;
}

template <typename T>
__device__ __forceinline__ T pivotFloor();
template <>
__device__ __forceinline__ double pivotFloor<double>() { return 1e-12; }
template <>
__device__ __forceinline__ float pivotFloor<float>() { return 1e-6f; }

// one lane group's sum over pairs q in [q0, q1) of lu[a] * rhs[c] for its system (serial in q)
template <typename T>
__device__ __forceinline__ T dotSerial(const T* __restrict__ lu, const T* __restrict__ rhs, const int2* __restrict__ pr,
                                       int64_t q0, int64_t q1, size_t B, int s) {
    T acc = T(0);
    int64_t q = q0;
    for (; q + 4 <= q1; q += 4) {
        const int2 a0 = __ldg(pr + q), a1 = __ldg(pr + q + 1), a2 = __ldg(pr + q + 2), a3 = __ldg(pr + q + 3);
        const T l0 = lu[a0.x * B + s], r0 = rhs[a0.y * B + s];
        const T l1 = lu[a1.x * B + s], r1 = rhs[a1.y * B + s];
        const T l2 = lu[a2.x * B + s], r2 = rhs[a2.y * B + s];
        const T l3 = lu[a3.x * B + s], r3 = rhs[a3.y * B + s];
        acc += l0 * r0;
        acc += l1 * r1;
        acc += l2 * r2;
        acc += l3 * r3;
    }
    for (; q < q1; q++) {
        const int2 a = __ldg(pr + q);
        acc += lu[a.x * B + s] * rhs[a.y * B + s];
    }
    return acc;
}

// Work descriptors (one int4 per schedule position, so that a piece of work costs one 16-byte load before its
// pairs): an entry of the factorisation or the forward substitution is {slot (or y index), first pair, end of
// pairs, kind | hasA << 2 | node << 3}; a node of the backward substitution is {node, LU base, |U row|, first
// row index}.
__device__ __forceinline__ int descKind(const int4& d) { return d.w & 3; }
__device__ __forceinline__ bool descHasA(const int4& d) { return (d.w >> 2) & 1; }
__device__ __forceinline__ int descNode(const int4& d) { return d.w >> 3; }

// How a piece of work is shared: one lane alone (serial sums: a lane group's short piece in the batched layouts, a
// thread's own piece in the one-system walks) or the whole warp (pair lanes).
enum PieceMode { kModeThread = 0, kModeWarp = 2 };

// One entry of the fused factorisation: A - sum(left * right), divided by the node's pivot for lower entries;
// the diagonal's result is the pivot (kept in its own array: the diagonal slot keeps A(k, k)). The value the entry
// starts from and its pivot are loaded before the sum, beside its operands.
template <typename T, int M>
__device__ __forceinline__ void factorPiece(const DevGrid& g, const DevBatch& b, const int4 d, int s, bool act) {
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    T* y = (T*)b.y;
    const int kind = descKind(d);
    const int slot = d.x;
    const int node = descNode(d);
    const int64_t q0 = d.y, q1 = d.z;
    const T a = kind == kFwd ? y[slot * B + s] : (descHasA(d) ? lu[slot * B + s] : T(0));
    const T pv = kind == kLower ? ((const T*)b.piv)[node * B + s] : T(1);
    const T* rhs = kind == kFwd ? y : lu;
    const T dot = M == kModeWarp ? dotSP<T>(lu, rhs, g.pairs, q0, q1, B, s) : dotSerial<T>(lu, rhs, g.pairs, q0, q1, B, s);
    const bool writer = M != kModeWarp || (threadIdx.x & 31) < Lay<T>::S;
    T v = a - dot;
    if (kind == kFwd) {
        if (writer) y[slot * B + s] = v;
        return;
    }
    if (kind == kDiag) {
        const T fl = pivotFloor<T>() * (fabs(a) > T(1) ? fabs(a) : T(1));
        if (!(fabs(v) > fl)) {  // static pivot collapsed (or NaN): perturb, flag, keep going
            if (act && writer) atomicOr(&b.flags[s], kFlagPivotPerturbed);
            v = (v < T(0)) ? -fl : fl;
        }
        if (writer) ((T*)b.piv)[node * B + s] = v;
        return;
    }
    if (kind == kLower) v = v / pv;
    if (writer) lu[slot * B + s] = v;
}
template <typename T>
__device__ __forceinline__ void factorEntry(const DevGrid& g, const DevBatch& b, const int4 d, int s, bool act, bool wide) {
    if (wide) factorPiece<T, kModeWarp>(g, b, d, s, act);
    else factorPiece<T, kModeThread>(g, b, d, s, act);
}

// backward substitution of a node: x(k) = (y(k) - sum U(k, r) x(r)) / U(k, k), in place
template <typename T, int M>
__device__ __forceinline__ void backwardPiece(const DevGrid& g, const DevBatch& b, T* y, const int4 d, int s) {
    constexpr int S = Lay<T>::S, P = Lay<T>::P;
    const size_t B = (size_t)b.B;
    const T* lu = (const T*)b.lu;
    const int k = d.x;
    const int64_t base = d.y;
    const int c = d.z;
    const int* rows = g.pRows + d.w;
    const T yk = y[k * B + s], pk = ((const T*)b.piv)[k * B + s];
    T acc = T(0);
    if (M == kModeWarp) {
        const int lane = threadIdx.x & 31;
        const int pl = lane / S;
        for (int t0 = 0; t0 < c; t0 += 32) {
            const int cnt = min(32, c - t0);
            const int mine = lane < cnt ? __ldg(rows + t0 + lane) : 0;
            const int uMax = (cnt + P - 1) / P;
            for (int v = 0; v < uMax; v++) {
                const int src = pl + P * v;
                const int r = __shfl_sync(0xffffffffu, mine, src);
                if (src < cnt) acc += lu[(base + 1 + t0 + src) * B + s] * y[r * B + s];
            }
        }
#pragma unroll
        for (int off = S; off < 32; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    } else {
        int t = 0;
        for (; t + 4 <= c; t += 4) {
            const int r0 = __ldg(rows + t), r1 = __ldg(rows + t + 1), r2 = __ldg(rows + t + 2), r3 = __ldg(rows + t + 3);
            const T u0 = lu[(base + 1 + t) * B + s], x0 = y[r0 * B + s];
            const T u1 = lu[(base + 2 + t) * B + s], x1 = y[r1 * B + s];
            const T u2 = lu[(base + 3 + t) * B + s], x2 = y[r2 * B + s];
            const T u3 = lu[(base + 4 + t) * B + s], x3 = y[r3 * B + s];
            acc += u0 * x0;
            acc += u1 * x1;
            acc += u2 * x2;
            acc += u3 * x3;
        }
        for (; t < c; t++) acc += lu[(base + 1 + t) * B + s] * y[__ldg(rows + t) * B + s];
    }
    const T xk = (yk - acc) / pk;
    if (M != kModeWarp || (threadIdx.x & 31) < S) y[k * B + s] = xk;
}
template <typename T>
__device__ __forceinline__ void backwardNode(const DevGrid& g, const DevBatch& b, T* y, const int4 d, int s, bool wide) {
    if (wide) backwardPiece<T, kModeWarp>(g, b, y, d, s);
    else backwardPiece<T, kModeThread>(g, b, y, d, s);
}

// forward substitution of a second right-hand side v: v(k) -= sum L(k, j) v(j), with node k's forward entry
template <typename T, int M>
__device__ __forceinline__ void forwardPiece(const DevGrid& g, const DevBatch& b, T* v, const int4 d, int s) {
    const size_t B = (size_t)b.B;
    const int k = descNode(d);
    const int64_t q0 = d.y, q1 = d.z;
    const T* lu = (const T*)b.lu;
    const T vk = v[k * B + s];
    const T dot = M == kModeWarp ? dotSP<T>(lu, v, g.pairs, q0, q1, B, s) : dotSerial<T>(lu, v, g.pairs, q0, q1, B, s);
    const T r = vk - dot;
    if (M != kModeWarp || (threadIdx.x & 31) < Lay<T>::S) v[k * B + s] = r;
}
template <typename T>
__device__ __forceinline__ void forwardEntry(const DevGrid& g, const DevBatch& b, T* v, const int4 d, int s, bool wide) {
    if (wide) forwardPiece<T, kModeWarp>(g, b, v, d, s);
    else forwardPiece<T, kModeThread>(g, b, v, d, s);
}

// the system of this lane in a warp of group `grp`
template <typename T>
__device__ __forceinline__ int laneSystem(int grp) { return grp * Lay<T>::S + ((threadIdx.x & 31) % Lay<T>::S); }

// Run one work item: a wide piece by the whole warp, or up to `count` short pieces over the lane groups.
template <typename T, typename F>
__device__ __forceinline__ void runItem(const int4* __restrict__ desc, const int* __restrict__ items, int it, F&& f) {
    const int start = __ldg(items + 2 * it), count = __ldg(items + 2 * it + 1);
    if (count < 0) {
        f(__ldg(desc + start), true);
    } else {
        for (int p = (threadIdx.x & 31) / Lay<T>::S; p < count; p += Lay<T>::P) f(__ldg(desc + start + p), false);
    }
}

enum WhichWork { kWorkFactor = 0, kWorkBackward = 1, kWorkForward = 2 };

template <typename T, int W>
__device__ __forceinline__ void doItem(const DevGrid& g, const DevBatch& b, T* vec, int it, int s, bool act) {
    if (W == kWorkFactor)
        runItem<T>(g.fDesc, g.fItems, it, [&](const int4 d, bool wide) { factorEntry<T>(g, b, d, s, act, wide); });
    else if (W == kWorkBackward)
        runItem<T>(g.bDesc, g.bItems, it, [&](const int4 d, bool wide) { backwardNode<T>(g, b, vec, d, s, wide); });
    else
        runItem<T>(g.vDesc, g.vItems, it, [&](const int4 d, bool wide) { forwardEntry<T>(g, b, vec, d, s, wide); });
}

// One level (or phase) of a schedule, items [i0, i1): block (32, 4), a warp per item, S systems per warp.
template <typename T, int W>
__global__ void __launch_bounds__(128, 10) k_level(DevGrid g, DevBatch b, T* vec, int i0, int i1) {
    const int it = i0 + blockIdx.x * 4 + threadIdx.y;
    const int s = laneSystem<T>(blockIdx.y);
    if (it >= i1) return;
    bool act = s < b.count && b.active[s];
    if (W != kWorkFactor && vec != (T*)b.y) act = act && b.refine[s];
    if (!__any_sync(0xffffffffu, act)) return;
    doItem<T, W>(g, b, vec, it, s, act);
}

// The narrow top of the elimination tree: one CTA per system group walks its levels itself, its warps
// sharing each level's items, with a block barrier between levels and phases (a CTA's systems are read and
// written by that CTA only, so no grid-wide synchronisation is needed; CTAs beyond one wave run later).
// `ptr` is the schedule's item pointer per level (per phase for the factorisation); `up` walks levels upward.
constexpr int kPersistWarps = 16;

template <typename T, int W>
__global__ void __launch_bounds__(32 * kPersistWarps) k_persistent(DevGrid g, DevBatch b, T* vec, int l0, int l1) {
    const int s = laneSystem<T>(blockIdx.x);
    bool act = s < b.count && b.active[s];
    if (W != kWorkFactor && vec != (T*)b.y) act = act && b.refine[s];
    if (!__syncthreads_or(act)) return;
    const int* ptr = W == kWorkFactor ? g.fLevelPtr : (W == kWorkBackward ? g.bLevelPtr : g.vLevelPtr);
    const int phases = W == kWorkFactor ? 2 : 1;
    for (int step = 0; step < l1 - l0; step++) {
        const int l = W == kWorkBackward ? l1 - 1 - step : l0 + step;
        for (int ph = 0; ph < phases; ph++) {
            const int i0 = ptr[phases * l + ph], i1 = ptr[phases * l + ph + 1];
            for (int it = i0 + threadIdx.y; it < i1; it += blockDim.y) doItem<T, W>(g, b, vec, it, s, act);
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Mixed precision: FP64 residual of the FP32 step, r = f - J dx, with J applied matrix-free from Y in FP64
// (the same H/N/M/L expressions as the fill). The correction solve of r with the same FP32 factors makes the
// step accurate to ~(kappa * 2^-24)^2, so the Newton path follows the FP64 path and stops where it stops.
template <typename T>
__device__ __forceinline__ void busResidual(const DevGrid& g, const DevBatch& b, int i, int s) {
    const size_t B = (size_t)b.B;
    const int et = g.qlim ? b.effType[i * B + s] : g.busType[i];
    const bool pId = g.qlim && (et == 3 || et == 0), qId = g.qlim && et != 1;  // identity rows (busMismatchJac)
    const int kp = g.busP[i], kq = g.busQ[i];
    if (kp < 0 && kq < 0) return;
    const T* dx = (const T*)b.y;
    T* z = (T*)b.z;
    if (!b.refine[s]) {
        if (kp >= 0) z[kp * B + s] = T(0);
        if (kq >= 0) z[kq * B + s] = T(0);
        return;
    }
    const double vmi = b.vm[i * B + s], vai = b.va[i * B + s];
    const int p0 = g.yRowPtr[i], p1 = g.yRowPtr[i + 1];
    // one pass: the injections, and the off-diagonal blocks applied to dx from the same sin/cos; the diagonal
    // blocks need P, Q and follow the loop
    CellOverride ovr(g, b.outage[s], p0);
    double pi = 0.0, qi = 0.0, jp = 0.0, jq = 0.0, Gd = 0.0, Bd = 0.0;
    for (int p = p0; p < p1; p++) {
        const int j = g.yCol[p];
        double G = g.yG[p], Bv = g.yB[p];
        ovr.at(g, p, G, Bv);
        double sn, cs;
        sincos(vai - b.va[j * B + s], &sn, &cs);
        const double vmj = b.vm[j * B + s];
        pi += vmj * (G * cs + Bv * sn);
        qi += vmj * (G * sn - Bv * cs);
        if (j == i) { Gd = G; Bd = Bv; continue; }
        const double H = vmi * vmj * (G * sn - Bv * cs);
        const double N = vmi * (G * cs + Bv * sn);
        const double M = -vmi * vmj * (G * cs + Bv * sn);
        const double L = vmi * (G * sn - Bv * cs);
        const int jP = g.busP[j], jQ = g.busQ[j];
        const double dth = jP >= 0 ? (double)dx[jP * B + s] : 0.0;
        const double dv = jQ >= 0 ? (double)dx[jQ * B + s] : 0.0;
        jp += H * dth + N * dv;
        jq += M * dth + L * dv;
    }
    {
        const double P = vmi * pi, Q = vmi * qi;
        const double sc = b.loadScale ? b.loadScale[i * B + s] : 1.0;
        double zdP, zdQ, zdPdV = 0.0, zdQdV = 0.0;
        const bool vcol = zipLoad(g, i, vmi, sc * g.pload[i], sc * g.qload[i], zdP, zdQ, zdPdV, zdQdV) && kq >= 0 && !qId;
        const double H = -Q - Bd * vmi * vmi;
        const double N = P / vmi + Gd * vmi + (vcol ? zdPdV : 0.0);
        const double M = P - Gd * vmi * vmi;
        const double L = Q / vmi - Bd * vmi + (vcol ? zdQdV : 0.0);
        const double dth = kp >= 0 ? (double)dx[kp * B + s] : 0.0;
        const double dv = kq >= 0 ? (double)dx[kq * B + s] : 0.0;
        jp += H * dth + N * dv;
        jq += M * dth + L * dv;
    }
    if (kp >= 0) z[kp * B + s] = pId ? T(0) : (T)(b.rhs64[kp * B + s] - jp);
    if (kq >= 0) z[kq * B + s] = qId ? T(0) : (T)(b.rhs64[kq * B + s] - jq);
}

template <typename T>
__global__ void __launch_bounds__(256) k_residual(DevGrid g, DevBatch b, const int* list, int nList) {
    const int lane = threadIdx.x, w = threadIdx.y;
    const int s = sysAt(blockIdx.y * 32 + lane, list, nList);
    const int i = blockIdx.x * 8 + w;
    if (i >= g.n || s < 0 || s >= b.count || !b.active[s]) return;
    busResidual<T>(g, b, i, s);
}

// ---------------------------------------------------------------------------------------------
// Few active systems (the last iterations of a batch, when almost every system has converged): one CTA per
// active system walks the levels itself, its threads taking the entries (nodes) of each level side by side,
// one dependent round of loads per level and phase. The system's LU is ~1 MB and stays in L2 across the
// levels; the per-level launches and their warps for 32-system groups are not needed here.
constexpr int kTailThreads = 1024;
// Two waves of k_tail CTAs (one 1024-thread CTA per SM). Measured on the 10,000-bus screen, where an iteration with
// ~220 of 5,000 systems left costs ~15 ms as a full-batch step and ~7 ms on this path: 148 (one wave) 22,200,
// 224 23,900, 296 24,200, 448 23,900 load flows/s in one run.
constexpr int kTailMaxSystems = 296;
constexpr int kCompactCap = 320;      // systems the compact workspace holds (kTailMaxSystems rounded up to 32)
constexpr double kMidCompactBelow = 0.7;  // full-batch step: compact once fewer than this share of its systems step

__global__ void k_collect_active(DevBatch b) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < b.count && b.active[s]) b.activeList[atomicAdd(b.activeCount, 1)] = s;
}

// Compaction of the few systems still stepping. Their state (voltages, load scalings, Newton control) moves
// into a workspace whose interleave stride is the number of systems rounded up to 32, so that a system's
// LU, right-hand sides and voltages span tens of MB instead of GB: the dependent loads of the level walk
// then hit L2. Everything else a step needs (Jacobian, LU, right-hand sides) is rebuilt from the state
// each iteration. Grid (ceil(n / 8), ceil(count / 32)), block (32, 8); position c of the compact batch
// holds system origin[c] of the full batch.
__device__ __forceinline__ void moveSystem(const DevBatch& from, int sf, const DevBatch& to, int st, int i, int n) {
    const size_t Bf = (size_t)from.B, Bt = (size_t)to.B;
    to.vm[i * Bt + st] = from.vm[i * Bf + sf];
    to.va[i * Bt + st] = from.va[i * Bf + sf];
    if (from.loadScale && to.loadScale) const_cast<double*>(to.loadScale)[i * Bt + st] = from.loadScale[i * Bf + sf];
    if (from.qState && to.qState) {
        to.effType[i * Bt + st] = from.effType[i * Bf + sf];
        to.qspecSys[i * Bt + st] = from.qspecSys[i * Bf + sf];
        to.pinned[i * Bt + st] = from.pinned[i * Bf + sf];
        to.reverted[i * Bt + st] = from.reverted[i * Bf + sf];
        if (i == 0) {
            to.passIter[st] = from.passIter[sf];
            to.qPass[st] = from.qPass[sf];
            to.qState[st] = from.qState[sf];
        }
    }
    if (i != 0) return;
    to.maxMis[st] = from.maxMis[sf];
    to.maxDx[st] = from.maxDx[sf];
    to.startMis[st] = from.startMis[sf];
    if (from.beforeLast && to.beforeLast) to.beforeLast[st] = from.beforeLast[sf];
    to.finalMis[st] = from.finalMis[sf];
    to.status[st] = from.status[sf];
    to.iters[st] = from.iters[sf];
    to.convIters[st] = from.convIters[sf];
    to.active[st] = from.active[sf];
    to.flags[st] = from.flags[sf];
    const_cast<int*>(to.outage)[st] = from.outage[sf];
    if (from.refine && to.refine) to.refine[st] = from.refine[sf];
    if (from.ovBus && to.ovBus) {
        for (int q = 0; q < 2; q++) {
            const_cast<int*>(to.ovBus)[2 * st + q] = from.ovBus[2 * sf + q];
            const_cast<int*>(to.ovType)[2 * st + q] = from.ovType[2 * sf + q];
            const_cast<double*>(to.ovVm)[2 * st + q] = from.ovVm[2 * sf + q];
        }
        const_cast<int*>(to.specBus)[st] = from.specBus[sf];
        const_cast<double*>(to.specDp)[st] = from.specDp[sf];
        const_cast<double*>(to.specDq)[st] = from.specDq[sf];
        const_cast<double*>(to.specQmin)[st] = from.specQmin[sf];
        const_cast<double*>(to.specQmax)[st] = from.specQmax[sf];
    }
}

// The batched linear solve's inputs into the workspace: A's stored entries into their LU slots, b into the
// right-hand side in pivot order. vals / rhs are system-major ([cnt][nnz], [cnt][n]); grid (ceil(max(nnz, n) / 8),
// B / 32), block (32, 8).
__global__ void k_load_matrix(DevBatch b, int cnt, int nnz, int n, const int* __restrict__ aSlot,
                              const int* __restrict__ pinv, const double* __restrict__ vals,
                              const double* __restrict__ rhs) {
    const int s = blockIdx.y * 32 + threadIdx.x, q = blockIdx.x * 8 + threadIdx.y;
    if (s >= b.B) return;
    const size_t B = (size_t)b.B;
    if (q == 0) { b.active[s] = s < cnt; b.flags[s] = 0; }
    if (s >= cnt) return;
    if (q < nnz) ((double*)b.lu)[(size_t)aSlot[q] * B + s] = vals[(size_t)s * nnz + q];
    if (q < n) ((double*)b.y)[(size_t)pinv[q] * B + s] = rhs[(size_t)s * n + q];
}

__global__ void k_gather(DevBatch full, DevBatch compact, const int* origin, int n) {
    const int c = blockIdx.y * 32 + threadIdx.x, i = blockIdx.x * 8 + threadIdx.y;
    if (c >= compact.count || i >= n) return;
    moveSystem(full, origin[c], compact, c, i, n);
}

// pairs[c] = (position in `from`, position in `to`): grid (ceil(n / 8), ceil(nPairs / 32)), block (32, 8).
__global__ void k_move_listed(DevBatch from, DevBatch to, const int2* pairs, int nPairs, int n) {
    const int c = blockIdx.y * 32 + threadIdx.x, i = blockIdx.x * 8 + threadIdx.y;
    if (c >= nPairs || i >= n) return;
    const int2 p = pairs[c];
    moveSystem(from, p.x, to, p.y, i, n);
}

__global__ void k_scatter(DevBatch compact, DevBatch full, const int* origin, int n) {
    const int c = blockIdx.y * 32 + threadIdx.x, i = blockIdx.x * 8 + threadIdx.y;
    if (c >= compact.count || i >= n) return;
    moveSystem(compact, c, full, origin[c], i, n);
}

// one system, the whole warp: lanes take pairs q0 + lane, q0 + lane + 32, ...; four pairs per lane are
// in flight at once (their index loads, then their eight value loads), then a fixed butterfly sum
template <typename T>
__device__ __forceinline__ T dotWarp1(const T* __restrict__ lu, const T* __restrict__ rhs, const int2* __restrict__ pr,
                                      int64_t q0, int64_t q1, size_t B, int s) {
    constexpr int U = 4;
    T acc = T(0);
    // the next round's index pairs are loaded while this round's operands are in flight
    int2 an[U];
    {
        const int64_t q = q0 + (threadIdx.x & 31);
#pragma unroll
        for (int u = 0; u < U; u++) an[u] = q + 32 * u < q1 ? __ldg(pr + q + 32 * u) : make_int2(-1, -1);
    }
    for (int64_t q = q0 + (threadIdx.x & 31); q < q1; q += 32 * U) {
        int2 a[U];
#pragma unroll
        for (int u = 0; u < U; u++) a[u] = an[u];
        if (q + 32 * U < q1) {
#pragma unroll
            for (int u = 0; u < U; u++) an[u] = q + 32 * (U + u) < q1 ? __ldg(pr + q + 32 * (U + u)) : make_int2(-1, -1);
        }
        T l[U], r[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool ok = a[u].x >= 0;
            l[u] = ok ? lu[a[u].x * B + s] : T(0);
            r[u] = ok ? rhs[a[u].y * B + s] : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) acc += l[u] * r[u];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    return acc;
}

// The few-systems path's wide pieces: one system, one warp.
template <typename T>
__device__ __forceinline__ void factorEntryWarp1(const DevGrid& g, const DevBatch& b, const int4 d, int s) {
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    T* y = (T*)b.y;
    const int kind = descKind(d), slot = d.x, node = descNode(d);
    const T dot = dotWarp1<T>(lu, kind == kFwd ? y : lu, g.pairs, d.y, d.z, B, s);
    if ((threadIdx.x & 31) != 0) return;
    if (kind == kFwd) { y[slot * B + s] -= dot; return; }
    const T a = descHasA(d) ? lu[slot * B + s] : T(0);
    T v = a - dot;
    if (kind == kDiag) {
        const T fl = pivotFloor<T>() * (fabs(a) > T(1) ? fabs(a) : T(1));
        if (!(fabs(v) > fl)) { atomicOr(&b.flags[s], kFlagPivotPerturbed); v = (v < T(0)) ? -fl : fl; }
        ((T*)b.piv)[node * B + s] = v;
        return;
    }
    if (kind == kLower) v = v / ((const T*)b.piv)[node * B + s];
    lu[slot * B + s] = v;
}

template <typename T>
__device__ __forceinline__ void backwardNodeWarp1(const DevGrid& g, const DevBatch& b, T* y, const int4 d, int s) {
    const size_t B = (size_t)b.B;
    const T* lu = (const T*)b.lu;
    const int k = d.x;
    const int64_t base = d.y;
    const int c = d.z;
    const int* rows = g.pRows + d.w;
    constexpr int U = 4;
    T acc = T(0);
    for (int t = threadIdx.x & 31; t < c; t += 32 * U) {
        int r[U];
#pragma unroll
        for (int u = 0; u < U; u++) r[u] = t + 32 * u < c ? __ldg(rows + t + 32 * u) : -1;
        T uu[U], x[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool ok = r[u] >= 0;
            uu[u] = ok ? lu[(base + 1 + t + 32 * u) * B + s] : T(0);
            x[u] = ok ? y[r[u] * B + s] : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) acc += uu[u] * x[u];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) y[k * B + s] = (y[k * B + s] - acc) / ((const T*)b.piv)[k * B + s];
}

template <typename T>
__device__ __forceinline__ void forwardEntryWarp1(const DevGrid& g, const DevBatch& b, T* v, const int4 d, int s) {
    const size_t B = (size_t)b.B;
    const int k = descNode(d);
    const T dot = dotWarp1<T>((const T*)b.lu, v, g.pairs, d.y, d.z, B, s);
    if ((threadIdx.x & 31) == 0) v[k * B + s] -= dot;
}

// One system, a group of G lanes of a warp (mask: the group's lanes): lane j of the group takes pairs q0 + j,
// q0 + j + G, ..., four at a time in flight; a fixed butterfly over the group completes the sum in every lane.
template <typename T, int G>
__device__ __forceinline__ T dotGroup(const T* __restrict__ lu, const T* __restrict__ rhs, const int2* __restrict__ pr,
                                      int q0, int q1, size_t B, int s, unsigned mask) {
    const int j = threadIdx.x & (G - 1);
    T acc = T(0);
    for (int q = q0 + j; q < q1; q += 4 * G) {
        int2 a[4];
#pragma unroll
        for (int u = 0; u < 4; u++) a[u] = q + u * G < q1 ? __ldg(pr + q + u * G) : make_int2(-1, -1);
        T l[4], r[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const bool ok = a[u].x >= 0;
            l[u] = ok ? lu[a[u].x * B + s] : T(0);
            r[u] = ok ? rhs[a[u].y * B + s] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) acc += l[u] * r[u];
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(mask, acc, off);
    return acc;
}

// the rest of a factorisation entry once its dot is known (by the one lane that writes it)
template <typename T>
__device__ __forceinline__ void factorFinish(const DevBatch& b, const int4 d, int s, T dot) {
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    const int kind = descKind(d), slot = d.x, node = descNode(d);
    if (kind == kFwd) {
        T* y = (T*)b.y;
        y[slot * B + s] -= dot;
        return;
    }
    const T a = descHasA(d) ? lu[slot * B + s] : T(0);
    T v = a - dot;
    if (kind == kDiag) {
        const T fl = pivotFloor<T>() * (fabs(a) > T(1) ? fabs(a) : T(1));
        if (!(fabs(v) > fl)) { atomicOr(&b.flags[s], kFlagPivotPerturbed); v = (v < T(0)) ? -fl : fl; }
        ((T*)b.piv)[node * B + s] = v;
        return;
    }
    if (kind == kLower) v = v / ((const T*)b.piv)[node * B + s];
    lu[slot * B + s] = v;
}

// a mid-length piece of a one-system walk by a group of G lanes
template <typename T, int W, int G>
__device__ __forceinline__ void groupPiece(const DevGrid& g, const DevBatch& b, T* vec, const int4 d, int s, unsigned mask) {
    const size_t B = (size_t)b.B;
    const bool lead = (threadIdx.x & (G - 1)) == 0;
    if (W == kWorkFactor) {
        const T* lu = (const T*)b.lu;
        const T dot = dotGroup<T, G>(lu, descKind(d) == kFwd ? (const T*)b.y : lu, g.pairs, d.y, d.z, B, s, mask);
        if (lead) factorFinish<T>(b, d, s, dot);
    } else if (W == kWorkForward) {
        const T dot = dotGroup<T, G>((const T*)b.lu, vec, g.pairs, d.y, d.z, B, s, mask);
        if (lead) vec[(size_t)descNode(d) * B + s] -= dot;
    } else {
        const T* lu = (const T*)b.lu;
        const int k = d.x, c = d.z;
        const int64_t base = d.y;
        const int* rows = g.pRows + d.w;
        const int j = threadIdx.x & (G - 1);
        T acc = T(0);
        for (int t = j; t < c; t += 4 * G) {
            int r[4];
#pragma unroll
            for (int u = 0; u < 4; u++) r[u] = t + u * G < c ? __ldg(rows + t + u * G) : -1;
            T uu[4], x[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const bool ok = r[u] >= 0;
                uu[u] = ok ? lu[(base + 1 + t + u * G) * B + s] : T(0);
                x[u] = ok ? vec[r[u] * B + s] : T(0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) acc += uu[u] * x[u];
        }
#pragma unroll
        for (int off = G / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(mask, acc, off);
        if (lead) vec[k * B + s] = (vec[k * B + s] - acc) / ((const T*)b.piv)[k * B + s];
    }
}

// One system, the whole block: every level (top down for the backward substitution) and phase of a schedule,
// the wide pieces a warp each, the short ones of more than 8 pairs a group of 8 lanes each, the rest a thread each,
// a block barrier between levels and phases.
template <typename T, int W>
__device__ __forceinline__ void walkLevels(const DevGrid& g, const DevBatch& b, T* vec, int s, int l0, int l1, int* queue) {
    const int* ptr = W == kWorkFactor ? g.fWorkPtr : (W == kWorkBackward ? g.bWorkPtr : g.vWorkPtr);
    const int4* desc = W == kWorkFactor ? g.fDesc : (W == kWorkBackward ? g.bDesc : g.vDesc);
    const int* midCnt = W == kWorkFactor ? g.fMid : (W == kWorkBackward ? g.bMid : g.vMid);
    const int* wide = W == kWorkFactor ? g.fWide : (W == kWorkBackward ? g.bWide : g.vWide);
    constexpr int G = 8;  // lanes per mid-length piece
    const int lane = threadIdx.x & 31, glead = lane & 24;
    const unsigned gmask = 0xFFu << glead;
    const int phases = W == kWorkFactor ? 2 : 1;
    // three shared counters per level and phase (wide, mid, rest), zeroed once per walk
    const int nq = 3 * phases * (l1 - l0);
    for (int k = threadIdx.x; k < nq; k += blockDim.x) queue[k] = 0;
    __syncthreads();
    for (int step = 0; step < l1 - l0; step++) {
        const int l = W == kWorkBackward ? l1 - 1 - step : l0 + step;
        for (int ph = 0; ph < phases; ph++) {
            const int i = phases * l + ph;
            int* q = queue + 3 * (phases * (l - l0) + ph);
            const int w0 = __ldg(ptr + i), w1 = __ldg(ptr + i + 1), nw = __ldg(wide + i), nm = __ldg(midCnt + i);
            // pieces are taken from the counters as warps, groups and threads come free: wide ones a warp each,
            // mid-length ones (longest first) a group of G lanes each, the rest a thread each, 32 per warp grab
            for (;;) {
                int w = 0;
                if (lane == 0) w = atomicAdd(q, 1);
                w = __shfl_sync(0xffffffffu, w, 0);
                if (w >= nw) break;
                const int4 x = __ldg(desc + w0 + w);
                if (W == kWorkFactor) factorEntryWarp1<T>(g, b, x, s);
                else if (W == kWorkBackward) backwardNodeWarp1<T>(g, b, vec, x, s);
                else forwardEntryWarp1<T>(g, b, vec, x, s);
            }
            for (;;) {
                int w = 0;
                if (lane == glead) w = atomicAdd(q + 1, 1);
                w = __shfl_sync(gmask, w, glead);
                if (w >= nm) break;
                groupPiece<T, W, G>(g, b, vec, __ldg(desc + w0 + nw + w), s, gmask);
            }
            const int nr = w1 - w0 - nw - nm;
            for (;;) {
                int w = 0;
                if (lane == 0) w = atomicAdd(q + 2, 32);
                w = __shfl_sync(0xffffffffu, w, 0);
                if (w >= nr) break;
                if (w + lane < nr) {
                    const int4 x = __ldg(desc + w0 + nw + nm + w + lane);
                    if (W == kWorkFactor) factorEntry<T>(g, b, x, s, true, false);
                    else if (W == kWorkBackward) backwardNode<T>(g, b, vec, x, s, false);
                    else forwardEntry<T>(g, b, vec, x, s, false);
                }
            }
            __syncthreads();
        }
    }
}

// ---- the top of the elimination tree in shared memory (levels >= L0 of the element size's DevTop) ----
template <typename T>
__device__ __forceinline__ const DevTop& topOf(const DevGrid& g) { return g.top[sizeof(T) == 4 ? 1 : 0]; }

// sum over pairs [q0, q1) of sm[x] * sm[y], both operands in shared memory: one warp (fixed butterfly), or one thread
template <typename T>
__device__ __forceinline__ T smDotWarp(const T* sm, const int2* __restrict__ pr, int q0, int q1) {
    T acc = T(0);
    for (int q = q0 + (int)(threadIdx.x & 31); q < q1; q += 32) {
        const int2 p = __ldg(pr + q);
        acc += sm[p.x] * sm[p.y];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    return acc;
}

template <typename T>
__device__ __forceinline__ T smDotSerial(const T* sm, const int2* __restrict__ pr, int q0, int q1) {
    T acc = T(0);
    int q = q0;
    for (; q + 4 <= q1; q += 4) {
        const int2 a0 = __ldg(pr + q), a1 = __ldg(pr + q + 1), a2 = __ldg(pr + q + 2), a3 = __ldg(pr + q + 3);
        acc += sm[a0.x] * sm[a0.y];
        acc += sm[a1.x] * sm[a1.y];
        acc += sm[a2.x] * sm[a2.y];
        acc += sm[a3.x] * sm[a3.y];
    }
    for (; q < q1; q++) {
        const int2 a = __ldg(pr + q);
        acc += sm[a.x] * sm[a.y];
    }
    return acc;
}

// Top entries of `list` (the first nWide a warp each, the rest a thread each) start in shared memory from their
// value (the right-hand side `rhs` for a forward entry, else A or 0) minus their external pairs, read from global.
template <typename T>
__device__ __forceinline__ void topLoad(const DevGrid& g, const DevBatch& b, const DevTop& t, T* sm, const T* rhs, int s,
                                        const int* list, int nWide, int n) {
    const size_t B = (size_t)b.B;
    const T* lu = (const T*)b.lu;
    const int warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
    for (int q = warp; q < nWide; q += nWarps) {
        const int ti = __ldg(list + q);
        const int e = __ldg(t.ent + ti);
        const bool fwd = g.entKind[e] == kFwd;
        const T ext = dotWarp1<T>(lu, fwd ? rhs : lu, t.extPairs, __ldg(t.extPtr + ti), __ldg(t.extPtr + ti + 1), B, s);
        if ((threadIdx.x & 31) == 0) {
            const T base = fwd ? rhs[(size_t)g.entNode[e] * B + s] : (g.entHasA[e] ? lu[(size_t)g.entSlot[e] * B + s] : T(0));
            sm[__ldg(t.entSm + ti)] = base - ext;
        }
    }
    for (int q = nWide + (int)threadIdx.x; q < n; q += (int)blockDim.x) {
        const int ti = __ldg(list + q);
        const int e = __ldg(t.ent + ti);
        const bool fwd = g.entKind[e] == kFwd;
        const T ext = dotSerial<T>(lu, fwd ? rhs : lu, t.extPairs, __ldg(t.extPtr + ti), __ldg(t.extPtr + ti + 1), B, s);
        const T base = fwd ? rhs[(size_t)g.entNode[e] * B + s] : (g.entHasA[e] ? lu[(size_t)g.entSlot[e] * B + s] : T(0));
        sm[__ldg(t.entSm + ti)] = base - ext;
    }
}

// the last step of a top entry of the factorisation: its value minus its internal dot; the pivot of a diagonal
// (perturbed to the floor of |A(k, k)| when it collapses), a lower entry divided by its node's pivot
template <typename T>
__device__ __forceinline__ void topFinish(const DevGrid& g, const DevBatch& b, const DevTop& t, T* sm, int ti, T dot, int s) {
    const int e = __ldg(t.ent + ti);
    const int kind = g.entKind[e];
    const int idx = __ldg(t.entSm + ti);
    T v = sm[idx] - dot;
    if (kind == kDiag) {
        const T a = g.entHasA[e] ? ((const T*)b.lu)[(size_t)g.entSlot[e] * b.B + s] : T(0);
        const T fl = pivotFloor<T>() * (fabs(a) > T(1) ? fabs(a) : T(1));
        if (!(fabs(v) > fl)) {
            atomicOr(&b.flags[s], kFlagPivotPerturbed);
            v = (v < T(0)) ? -fl : fl;
        }
    } else if (kind == kLower) {
        v = v / sm[__ldg(t.smemBase + g.entNode[e])];
    }
    sm[idx] = v;
}

// One system, the whole block: the fused factorisation + forward substitution. Levels below L0 walk global
// memory; the top is loaded into shared memory `sm` (external pairs applied on the way), walked there, and
// written back (U and L to the LU, pivots to piv, the forward-substituted right-hand side to y).
template <typename T>
__device__ void factorSystem(const DevGrid& g, const DevBatch& b, int s, T* sm, bool useTop, int* queue) {
    const DevTop& t = topOf<T>(g);
    walkLevels<T, kWorkFactor>(g, b, (T*)b.y, s, 0, useTop ? t.L0 : g.nLevels, queue);
    if (!useTop || t.L0 >= g.nLevels) return;
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    T* y = (T*)b.y;
    T* piv = (T*)b.piv;
    const int warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5, lane = threadIdx.x & 31;
    topLoad<T>(g, b, t, sm, y, s, t.loadList, t.loadWide, t.nLoad);
    __syncthreads();
    const int nTop = g.nLevels - t.L0;
    for (int i = 0; i < 2 * nTop; i++) {
        const int w0 = __ldg(t.fWalkPtr + i), w1 = __ldg(t.fWalkPtr + i + 1), nw = __ldg(t.fWalkWide + i);
        for (int w = w0 + warp; w < w0 + nw; w += nWarps) {
            const int ti = __ldg(t.fWalk + w);
            const T dot = smDotWarp<T>(sm, t.intPairs, __ldg(t.intPtr + ti), __ldg(t.intPtr + ti + 1));
            if (lane == 0) topFinish<T>(g, b, t, sm, ti, dot, s);
        }
        for (int w = w0 + nw + (int)threadIdx.x; w < w1; w += (int)blockDim.x) {
            const int ti = __ldg(t.fWalk + w);
            topFinish<T>(g, b, t, sm, ti, smDotSerial<T>(sm, t.intPairs, __ldg(t.intPtr + ti), __ldg(t.intPtr + ti + 1)), s);
        }
        __syncthreads();
    }
    for (int q = threadIdx.x; q < t.nSlots; q += blockDim.x) {
        const int node = __ldg(t.slotDiagNode + q);
        if (node >= 0) piv[(size_t)node * B + s] = sm[q];
        else lu[(size_t)__ldg(t.slotGlobal + q) * B + s] = sm[q];
    }
    for (int i = threadIdx.x; i < t.nNodes; i += blockDim.x) y[(size_t)__ldg(t.nodes + i) * B + s] = sm[t.nSlots + i];
    __syncthreads();
}

// One system, the whole block: backward substitution of `vec` in place, the top in shared memory first.
template <typename T>
__device__ void backwardSystem(const DevGrid& g, const DevBatch& b, T* vec, int s, T* sm, bool useTop, int* queue) {
    const DevTop& t = topOf<T>(g);
    const int L0 = useTop ? t.L0 : g.nLevels;
    if (L0 < g.nLevels) {
        const size_t B = (size_t)b.B;
        const T* lu = (const T*)b.lu;
        const T* piv = (const T*)b.piv;
        const int warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5, lane = threadIdx.x & 31;
        for (int q = threadIdx.x; q < t.nSlots; q += blockDim.x) {
            const int node = __ldg(t.slotDiagNode + q);
            sm[q] = node >= 0 ? piv[(size_t)node * B + s] : lu[(size_t)__ldg(t.slotGlobal + q) * B + s];
        }
        for (int i = threadIdx.x; i < t.nNodes; i += blockDim.x) sm[t.nSlots + i] = vec[(size_t)__ldg(t.nodes + i) * B + s];
        __syncthreads();
        const int nTop = g.nLevels - t.L0;
        for (int lt = nTop - 1; lt >= 0; lt--) {
            const int w0 = __ldg(t.bWalkPtr + lt), w1 = __ldg(t.bWalkPtr + lt + 1), nw = __ldg(t.bWalkWide + lt);
            for (int w = w0 + warp; w < w0 + nw; w += nWarps) {
                const int ni = __ldg(t.bWalk + w);
                const int k = __ldg(t.nodes + ni), base = __ldg(t.smemBase + k), c = g.luCnt[k];
                const int* rows = t.bRowSm + __ldg(t.bRowPtr + ni);
                T acc = T(0);
                for (int u = lane; u < c; u += 32) acc += sm[base + 1 + u] * sm[__ldg(rows + u)];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
                if (lane == 0) sm[t.nSlots + ni] = (sm[t.nSlots + ni] - acc) / sm[base];
            }
            for (int w = w0 + nw + (int)threadIdx.x; w < w1; w += (int)blockDim.x) {
                const int ni = __ldg(t.bWalk + w);
                const int k = __ldg(t.nodes + ni), base = __ldg(t.smemBase + k), c = g.luCnt[k];
                const int* rows = t.bRowSm + __ldg(t.bRowPtr + ni);
                T acc = T(0);
                for (int u = 0; u < c; u++) acc += sm[base + 1 + u] * sm[__ldg(rows + u)];
                sm[t.nSlots + ni] = (sm[t.nSlots + ni] - acc) / sm[base];
            }
            __syncthreads();
        }
        for (int i = threadIdx.x; i < t.nNodes; i += blockDim.x) vec[(size_t)__ldg(t.nodes + i) * B + s] = sm[t.nSlots + i];
        __syncthreads();
    }
    walkLevels<T, kWorkBackward>(g, b, vec, s, 0, L0, queue);
}

// One system, the whole block: forward substitution of a second right-hand side `vec` in place.
template <typename T>
__device__ void forwardSystem(const DevGrid& g, const DevBatch& b, T* vec, int s, T* sm, bool useTop, int* queue) {
    const DevTop& t = topOf<T>(g);
    walkLevels<T, kWorkForward>(g, b, vec, s, 0, useTop ? t.L0 : g.nLevels, queue);
    if (!useTop || t.L0 >= g.nLevels) return;
    const size_t B = (size_t)b.B;
    const T* lu = (const T*)b.lu;
    const int warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int q = threadIdx.x; q < t.nSlots; q += blockDim.x) sm[q] = lu[(size_t)__ldg(t.slotGlobal + q) * B + s];
    topLoad<T>(g, b, t, sm, vec, s, t.fwdLoadList, t.fwdLoadWide, t.nFwdLoad);
    __syncthreads();
    const int nTop = g.nLevels - t.L0;
    for (int lt = 0; lt < nTop; lt++) {
        const int w0 = __ldg(t.vWalkPtr + lt), w1 = __ldg(t.vWalkPtr + lt + 1), nw = __ldg(t.vWalkWide + lt);
        for (int w = w0 + warp; w < w0 + nw; w += nWarps) {
            const int ti = __ldg(t.vWalk + w);
            const T dot = smDotWarp<T>(sm, t.intPairs, __ldg(t.intPtr + ti), __ldg(t.intPtr + ti + 1));
            if (lane == 0) sm[__ldg(t.entSm + ti)] -= dot;
        }
        for (int w = w0 + nw + (int)threadIdx.x; w < w1; w += (int)blockDim.x) {
            const int ti = __ldg(t.vWalk + w);
            sm[__ldg(t.entSm + ti)] -= smDotSerial<T>(sm, t.intPairs, __ldg(t.intPtr + ti), __ldg(t.intPtr + ti + 1));
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < t.nNodes; i += blockDim.x) vec[(size_t)__ldg(t.nodes + i) * B + s] = sm[t.nSlots + i];
    __syncthreads();
}

// Dynamic shared memory of the one-system kernels: the top part of the grid's schedule (when used), then the piece
// counters of the level walks.
extern __shared__ __align__(16) unsigned char gsTopSmem[];

// Levels [l0, l1) of a schedule for the listed systems, one CTA each (the wide levels below l0 run as per-level
// launches over the same batch). Dynamic shared memory: the walk's piece counters (QueueBytes).
template <typename T, int W>
__global__ void __launch_bounds__(kTailThreads) k_tail(DevGrid g, DevBatch b, T* vec, int l0, int l1) {
    const int s = b.activeList[blockIdx.x];
    if (W != kWorkFactor && vec != (T*)b.y && !b.refine[s]) return;  // uniform across the block
    walkLevels<T, W>(g, b, vec, s, l0, l1, reinterpret_cast<int*>(gsTopSmem));
}

// shared memory of the piece counters of a walk over every level of a grid
inline size_t QueueBytes(int nLevels) { return (size_t)6 * nLevels * sizeof(int); }

}  // namespace gs
#include "gs_paired.cuh"
#include "gs_cluster.cuh"
#include "gs_pivot.cuh"
namespace gs {

// One step of the few systems of a batch (their list in b.activeList): factorisation, backward substitution and,
// in mixed precision, the FP64-residual refinement. With `cluster` every level runs as one cluster of CTAs per system
// (gs_cluster.cuh; 8 CTAs each for a handful of systems, fewer as they grow); otherwise levels below `lt` (many entries each) run as
// per-level launches over the batch, the levels above as one CTA per system.
template <typename T>
int64_t FewSystemsSolve(const DevGrid& g, const DevBatch& b, const Symbolic& s, int nActive, int lt, bool refine,
                        cudaStream_t st, cudaEvent_t afterFactor, bool cluster = false, bool paired = false) {
    int64_t launches = 0;
    const bool pk = paired && g.psLevels > 0;
    const int Lc = pk ? g.psLevels : s.nLevels;
    if (cluster && nActive <= kClusterMaxSystems && ClusterSmemBytes(Lc) <= kClusterSmemMax) {
        LaunchTailCluster<T, kWorkFactor>(g, b, (T*)b.y, 0, Lc, nActive, st, pk);
        if (afterFactor) cudaEventRecord(afterFactor, st);
        LaunchTailCluster<T, kWorkBackward>(g, b, (T*)b.y, 0, Lc, nActive, st, pk);
        launches += 2;
        if (refine) {
            k_residual<T><<<dim3((s.n + 7) / 8, (nActive + 31) / 32), dim3(32, 8), 0, st>>>(g, b, b.activeList, nActive);
            LaunchTailCluster<T, kWorkForward>(g, b, (T*)b.z, 0, Lc, nActive, st, pk);
            LaunchTailCluster<T, kWorkBackward>(g, b, (T*)b.z, 0, Lc, nActive, st, pk);
            launches += 3;
        }
        return launches;
    }
    const int groups = b.B / Lay<T>::S;
    const dim3 blk4(32, 4), blk8(32, 8);
    auto level = [&](auto kernel, T* vec, int i0, int i1) {
        if (i1 > i0) { kernel<<<dim3((i1 - i0 + 3) / 4, groups), blk4, 0, st>>>(g, b, vec, i0, i1); launches++; }
    };
    const auto& fp = s.factor.levelItemPtr;
    const auto& bp = s.backward.levelItemPtr;
    const auto& vp = s.forward.levelItemPtr;
    const int L = s.nLevels;
    const size_t qb = QueueBytes(L);
    auto backward = [&](T* vec) {
        k_tail<T, kWorkBackward><<<nActive, kTailThreads, qb, st>>>(g, b, vec, lt, L);
        launches++;
        for (int l = lt - 1; l >= 0; l--) level(k_level<T, kWorkBackward>, vec, bp[l], bp[l + 1]);
    };
    for (int l = 0; l < lt; l++) {
        level(k_level<T, kWorkFactor>, (T*)b.y, fp[2 * l], fp[2 * l + 1]);
        level(k_level<T, kWorkFactor>, (T*)b.y, fp[2 * l + 1], fp[2 * l + 2]);
    }
    k_tail<T, kWorkFactor><<<nActive, kTailThreads, qb, st>>>(g, b, (T*)b.y, lt, L);
    launches++;
    if (afterFactor) cudaEventRecord(afterFactor, st);
    backward((T*)b.y);
    if (refine) {
        k_residual<T><<<dim3((s.n + 7) / 8, (nActive + 31) / 32), blk8, 0, st>>>(g, b, b.activeList, nActive);
        for (int l = 0; l < lt; l++) level(k_level<T, kWorkForward>, (T*)b.z, vp[l], vp[l + 1]);
        k_tail<T, kWorkForward><<<nActive, kTailThreads, qb, st>>>(g, b, (T*)b.z, lt, L);
        launches += 2;
        backward((T*)b.z);
    }
    return launches;
}

// ---------------------------------------------------------------------------------------------
// 5. max |dx| per system, then the damped update.
template <typename T>
__global__ void __launch_bounds__(256) k_dxmax(DevGrid g, DevBatch b, int rowsPerBlock, int refine, const int* list,
                                               int nList) {
    const int lane = threadIdx.x, w = threadIdx.y;
    const int s = sysAt(blockIdx.y * 32 + lane, list, nList);
    const size_t B = (size_t)b.B;
    const T* y = (const T*)b.y;
    const T* z = (const T*)b.z;
    const int r0 = blockIdx.x * rowsPerBlock, r1 = min(g.m, r0 + rowsPerBlock);
    double mx = 0.0;
    bool bad = false;
    if (s >= 0 && s < b.count && b.active[s]) {
        for (int k = r0 + w; k < r1; k += 8) {
            const double v = (double)y[k * B + s] + (refine && b.refine[s] ? (double)z[k * B + s] : 0.0);
            bad |= !isfinite(v);
            mx = fmax(mx, fabs(v));
        }
    }
    __shared__ double red[8][32];
    __shared__ int redBad[8][32];
    red[w][lane] = mx;
    redBad[w][lane] = bad;
    __syncthreads();
    if (w == 0 && s >= 0 && s < b.count) {
        double m = red[0][lane];
        int anyBad = redBad[0][lane];
        for (int q = 1; q < 8; q++) { m = fmax(m, red[q][lane]); anyBad |= redBad[q][lane]; }
        if (m > 0.0) atomicMaxNonNeg(&b.maxDx[s], m);
        if (anyBad) atomicOr(&b.flags[s], kFlagStepBad);
    }
}

// the damped update of bus i of system s (the system's max |dx| is in maxDx); bus 0 counts the step
template <typename T>
__device__ __forceinline__ void busUpdate(const DevGrid& g, const DevBatch& b, int i, int s, int refine) {
    const size_t B = (size_t)b.B;
    const T* y = (const T*)b.y;
    const T* z = (const T*)b.z;
    refine = refine && b.refine[s];
    const double mx = __longlong_as_double((long long)b.maxDx[s]);
    const double damp = mx > kMaxUndampedStep ? kMaxUndampedStep / mx : 1.0;
    const int kp = g.busP[i], kq = g.busQ[i];
    if (kp >= 0) b.va[i * B + s] += damp * ((double)y[kp * B + s] + (refine ? (double)z[kp * B + s] : 0.0));
    if (kq >= 0) {
        double v = b.vm[i * B + s] + damp * ((double)y[kq * B + s] + (refine ? (double)z[kq * B + s] : 0.0));
        if (v < kVmFloorPu) v = kVmFloorPu;
        b.vm[i * B + s] = v;
    }
    if (i == 0) {
        b.iters[s] += 1;
        if (b.passIter) b.passIter[s] += 1;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_update(DevGrid g, DevBatch b, int refine, const int* list, int nList) {
    const int lane = threadIdx.x;
    const int s = sysAt(blockIdx.y * 32 + lane, list, nList);
    const int i = blockIdx.x * 8 + threadIdx.y;
    if (i >= g.n || s < 0 || s >= b.count || !b.active[s]) return;
    if (b.flags[s] & kFlagStepBad) return;
    if (b.qState && (b.qState[s] & kQSkipStep)) return;  // a new Q-limit pass starts from this state
    busUpdate<T>(g, b, i, s, refine);
}

// ---------------------------------------------------------------------------------------------
// start state: every system from the shared start (vm0/va0) or from a base state of one system.
// vmSys / vaSys ([n][B], may be null): a start state per system (the DC retry), else vmStart / vaStart for all.
__global__ void k_init(DevGrid g, DevBatch b, const double* vmStart, const double* vaStart, const double* vmSys,
                       const double* vaSys) {
    const int lane = threadIdx.x;
    const int s = blockIdx.y * 32 + lane;
    const int i = blockIdx.x * 8 + threadIdx.y;
    if (i >= g.n || s >= b.B) return;
    const size_t B = (size_t)b.B;
    double vm = vmSys ? vmSys[i * B + s] : (vmStart ? vmStart[i] : g.vm0[i]);
    double va = vaSys ? vaSys[i * B + s] : (vaStart ? vaStart[i] : g.va0[i]);
    // an element outage may change this bus's type in this system, and its set point or stored magnitude
    const int gt = g.busType[i];
    int et = gt;
    double ov = NAN;
    if (b.ovBus && s < b.count) {
        if (b.ovBus[2 * s] == i) { et = b.ovType[2 * s]; ov = b.ovVm[2 * s]; }
        else if (b.ovBus[2 * s + 1] == i) { et = b.ovType[2 * s + 1]; ov = b.ovVm[2 * s + 1]; }
    }
    // PV and reference magnitudes are set points whatever the start (NewtonShell.BuildBusSpec :467-469)
    if (et == 2 || et == 3) vm = isnan(ov) ? g.vm0[i] : ov;
    else if (!isnan(ov) && !vmSys && !vmStart) vm = ov;  // a bus that starts PQ here: its stored magnitude
    if (gt == 3 && et == 3) va = g.va0[i];
    b.vm[i * B + s] = vm;
    b.va[i * B + s] = va;
    if (b.qState) {
        b.effType[i * B + s] = et;
        double qs = 0.0;
        if (et == 1 && gt != 1) {  // left without units: Q is what the units left give, less the load
            const double qd = (b.loadScale ? b.loadScale[i * B + s] : 1.0) * g.qload[i];
            qs = ((b.specBus && b.specBus[s] == i) ? g.qgen[i] - b.specDq[s] : g.qgen[i]) - qd;
        }
        b.qspecSys[i * B + s] = qs;
        b.pinned[i * B + s] = 0;
        b.reverted[i * B + s] = 0;
        if (i == 0) { b.passIter[s] = 0; b.qPass[s] = 0; b.qState[s] = 0; }
    }
    if (i == 0) {
        b.maxMis[s] = 0ull;
        b.maxDx[s] = 0ull;
        b.startMis[s] = 0.0;
        if (b.beforeLast) b.beforeLast[s] = NAN;
        b.finalMis[s] = NAN;
        b.status[s] = s < b.count ? GS_PF_MAX_ITERATIONS : GS_PF_NOT_RUN;
        b.iters[s] = 0;
        b.convIters[s] = 0;
        if (b.refine) b.refine[s] = 0;
        b.active[s] = s < b.count ? 1 : 0;
        b.flags[s] = 0;
    }
}

// ---------------------------------------------------------------------------------------------
// Post-processing of converged systems (ContingencyAnalysis.ScreenStateCore :1150-1235): branch
// loading (NewtonShell.ComputeLineFlows :699-734), the thermal test (> 100 %), the voltage test against
// each bus's limits (per-bus or the 0.94 / 1.06 band, VoltageLimits.cs:28-67). Items are the branches in
// order, then the buses in order, which is the order of ContingencyResult.Details.
struct Classify {
    const double* lo;  // [n] effective lower limit
    const double* hi;
    uint8_t* code;     // [items][B]: 0 none, 1 overload, 2 under, 3 over, 4 boundary overload
    double* value;     // [items][B]
    unsigned long long* maxLoad;  // [B]
    unsigned long long* minVmNeg; // [B] max of (-Vm) stored as bits of (100 - Vm) (positive)
    unsigned long long* maxVm;    // [B]
    unsigned long long* worstBnd; // [B]
    int* chunkCount;   // [nChunks][B]
    int chunk;
    int postRating;    // enum gs_post_fault_rating: the rating of outage states
};

// From-end and to-end complex power of branch k in system s, pu (NewtonShell.ComputeLineFlows :699-734).
__device__ __forceinline__ void branchPower(const DevGrid& g, const DevBatch& b, int k, int s, double& sFr,
                                            double& sFi, double& sTr, double& sTi) {
    const size_t B = (size_t)b.B;
    const int f = g.brF[k], t = g.brT[k];
    double sf, cf, st, ct;
    sincos(b.va[f * B + s], &sf, &cf);
    sincos(b.va[t * B + s], &st, &ct);
    const double vfr = b.vm[f * B + s] * cf, vfi = b.vm[f * B + s] * sf;
    const double vtr = b.vm[t * B + s] * ct, vti = b.vm[t * B + s] * st;
    const double* y = g.brStamp + 8 * k;
    // iF = yff vf + yft vt ; iT = ytf vf + ytt vt
    const double ifr = y[0] * vfr - y[1] * vfi + y[4] * vtr - y[5] * vti;
    const double ifi = y[0] * vfi + y[1] * vfr + y[4] * vti + y[5] * vtr;
    const double itr = y[6] * vfr - y[7] * vfi + y[2] * vtr - y[3] * vti;
    const double iti = y[6] * vfi + y[7] * vfr + y[2] * vti + y[3] * vtr;
    // S = V conj(I)
    sFr = vfr * ifr + vfi * ifi; sFi = vfi * ifr - vfr * ifi;
    sTr = vtr * itr + vti * iti; sTi = vti * itr - vtr * iti;
}

// Items per system: the branches (thermal), the boundaries, then the buses (voltage), in the order the reference
// lists the violations (ScreenStateCore :1150-1235).
__global__ void k_classify(DevGrid g, DevBatch b, Classify c) {
    const int lane = threadIdx.x;
    const int s = blockIdx.y * 32 + lane;
    const int item = blockIdx.x * 8 + threadIdx.y;
    const int nItems = g.nbr + g.nBnd + g.n;
    if (item >= nItems || s >= b.count) return;
    const size_t B = (size_t)b.B;
    uint8_t code = 0;
    double val = 0.0;
    if (b.status[s] == GS_PF_CONVERGED) {
        const int o = b.outage[s];
        if (item < g.nbr) {
            const int k = item;
            if (g.brOn[k] && !branchOut(g, o, k)) {
                double sFr, sFi, sTr, sTi;
                branchPower(g, b, k, s, sFr, sFi, sTr, sTi);
                const double mva = fmax(hypot(sFr, sFi), hypot(sTr, sTi));
                // base_mva folded into the ratings (the host passes rating / base); an outage state may be judged
                // against RateB / RateC, falling back to RateA where that rating is 0 (:1273-1284)
                double r = g.rateA[k];
                if (c.postRating != GS_RATE_A && o >= 0) {
                    const double rx = c.postRating == GS_RATE_B ? g.rateB[k] : g.rateC[k];
                    if (rx > 0) r = rx;
                }
                val = r > 0 ? mva / r * 100.0 : 0.0;
                if (val > 0.0) atomicMaxNonNeg(&c.maxLoad[s], val);
                if (val > 100.0) code = 1;
            }
        } else if (item < g.nbr + g.nBnd) {
            // BoundaryAnalysis.EvaluateAfterOutage (Analysis/BoundaryAnalysis.cs:43-68): the signed sum of the members'
            // from-end MW; the outaged branch is not in the reduced model, an out-of-service one carries nothing
            const int q = item - g.nbr;
            double flow = 0.0;
            for (int e = g.bndPtr[q]; e < g.bndPtr[q + 1]; e++) {
                const int k = g.bndBranch[e];
                if (!g.brOn[k] || branchOut(g, o, k)) continue;
                double sFr, sFi, sTr, sTi;
                branchPower(g, b, k, s, sFr, sFi, sTr, sTi);
                flow += g.bndDir[e] * (sFr * g.baseMva);
            }
            const double lim = g.bndLimit[q];
            val = lim > 0 ? fabs(flow) / lim * 100.0 : 0.0;
            if (val > 0.0) atomicMaxNonNeg(&c.worstBnd[s], val);
            if (lim > 0 && fabs(flow) > lim) code = 4;
        } else {
            const int i = item - g.nbr - g.nBnd;
            if (!(g.qlim && b.effType[i * B + s] == 0)) {  // a removed bus is not in the reduced model
                val = b.vm[i * B + s];
                if (val < c.lo[i]) code = 2;
                else if (val > c.hi[i]) code = 3;
                atomicMaxNonNeg(&c.maxVm[s], val);
                atomicMaxNonNeg(&c.minVmNeg[s], 100.0 - val);
            }
        }
    }
    c.code[(size_t)item * B + s] = code;
    c.value[(size_t)item * B + s] = val;
    if (code) atomicAdd(&c.chunkCount[(size_t)(item / c.chunk) * B + s], 1);
}

// Ordered compaction: one warp per (chunk, 32 systems); each lane walks the chunk in item order.
__global__ void k_compact(DevGrid g, DevBatch b, Classify c, const int* chunkOffset, int* outKind, int* outElem,
                          double* outVal, const int* busId) {
    const int lane = threadIdx.x;
    const int s = blockIdx.y * 32 + lane;
    const int ch = blockIdx.x * 4 + threadIdx.y;
    const int nItems = g.nbr + g.nBnd + g.n;
    const int nChunks = (nItems + c.chunk - 1) / c.chunk;
    if (ch >= nChunks || s >= b.count) return;
    const size_t B = (size_t)b.B;
    int w = chunkOffset[(size_t)ch * B + s];
    const int e = min(nItems, (ch + 1) * c.chunk);
    for (int item = ch * c.chunk; item < e; item++) {
        const uint8_t code = c.code[(size_t)item * B + s];
        if (!code) continue;
        outKind[w] = code == 1 ? GS_VIOL_BRANCH_OVERLOAD
                   : code == 4 ? GS_VIOL_BOUNDARY_OVERLOAD
                   : (code == 2 ? GS_VIOL_UNDERVOLTAGE : GS_VIOL_OVERVOLTAGE);
        outElem[w] = code == 1 ? item : code == 4 ? item - g.nbr : busId[item - g.nbr - g.nBnd];
        outVal[w] = c.value[(size_t)item * B + s];
        w++;
    }
}

// Line flows of system 0 (single solve result).
__global__ void k_lineflows(DevGrid g, DevBatch b, double base, double* loading, double* sfo, double* sto) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.nbr) return;
    const size_t B = (size_t)b.B;
    if (!g.brOn[k]) {
        loading[k] = 0; sfo[2 * k] = sfo[2 * k + 1] = sto[2 * k] = sto[2 * k + 1] = 0;
        return;
    }
    const int f = g.brF[k], t = g.brT[k];
    double sf, cf, st, ct;
    sincos(b.va[f * B], &sf, &cf);
    sincos(b.va[t * B], &st, &ct);
    const double vfr = b.vm[f * B] * cf, vfi = b.vm[f * B] * sf;
    const double vtr = b.vm[t * B] * ct, vti = b.vm[t * B] * st;
    const double* y = g.brStamp + 8 * k;
    const double ifr = y[0] * vfr - y[1] * vfi + y[4] * vtr - y[5] * vti;
    const double ifi = y[0] * vfi + y[1] * vfr + y[4] * vti + y[5] * vtr;
    const double itr = y[6] * vfr - y[7] * vfi + y[2] * vtr - y[3] * vti;
    const double iti = y[6] * vfi + y[7] * vfr + y[2] * vti + y[3] * vtr;
    const double sFr = (vfr * ifr + vfi * ifi) * base, sFi = (vfi * ifr - vfr * ifi) * base;
    const double sTr = (vtr * itr + vti * iti) * base, sTi = (vti * itr - vtr * iti) * base;
    sfo[2 * k] = sFr; sfo[2 * k + 1] = sFi;
    sto[2 * k] = sTr; sto[2 * k + 1] = sTi;
    const double mva = fmax(hypot(sFr, sFi), hypot(sTr, sTi));
    const double r = g.rateA[k] * base;
    loading[k] = r > 0 ? mva / r * 100.0 : 0.0;
}

// FP64 self-test (GpuContext.cs:227-254): (1 + 2^-40) - 1 must be 2^-40 exactly.
__global__ void k_selftest(double* out) {
    volatile double one = 1.0;
    double e = ldexp(1.0, -40);
    out[0] = (one + e) - one;
}

}  // namespace gs

// =============================================================================================
// Host side.
namespace gs {

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) {
        if (p && bytes >= n) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        if (n == 0) n = 16;
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n; else p = nullptr;
        return e;
    }
    template <typename X> X* as() const { return reinterpret_cast<X*>(p); }
};

// Two events bracketing device work on one stream; ms() once both have completed.
struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    EventPair() = default;
    EventPair(const EventPair&) = delete;
    EventPair& operator=(const EventPair&) = delete;
    ~EventPair() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
    cudaError_t create() {
        cudaError_t e = cudaEventCreate(&a);
        return e == cudaSuccess ? cudaEventCreate(&b) : e;
    }
    float ms() const { float t = 0; cudaEventElapsedTime(&t, a, b); return t; }
};

struct Workspace {
    int B = 0;
    int precision = -1;
    DevBuf activeList, origin;  // origin: a compact batch position -> the system of the full batch
    DevBuf effType, qspecSys, pinned, reverted, qinj, passIter, qPass, qState;  // Q-limit enforcement
    DevBuf ovBus, ovType, ovVm, specBus, specDp, specDq, specQmin, specQmax;    // element outages
    bool ovOn = false;  // the element-outage arrays hold this call's systems
    DevBuf beforeLast;
    DevBuf vm, va, lu, piv, y, z, rhs64, refine, maxMis, maxDx, startMis, finalMis, status, iters, convIters, active, flags, outage,
        loadScale, activeCount;
    DevBuf code, value, maxLoad, minVmNeg, maxVmB, worstBnd, chunkCount, chunkOffset, outKind, outElem, outVal, pq;
    DevBuf startVm, startVa;
};

// The partial-pivoting re-solve of one grid (or matrix pattern): the matrix's cells by column (Symbolic::aColPtr,
// aRow, aSlot) on the device, and the factorisation scratch of up to `maxSys` systems with `cap` L and U entries each.
struct GpData {
    DevBuf colPtr, row, slot;
    DevBuf x, rowMax, xi, pstack, mark, pinv, lp, up, li, ui, lx, ux, result;
    int maxSys = 0;
    int64_t cap = 0;
    bool uploaded = false;
    // the iterative fallback (ILU(0) + BiCGSTAB) of the Newton step: the Jacobian in equation order and the Y cells'
    // stamps, and its scratch
    DevBuf jRowPtr, jCol, jSlot, jYcell, eqPinv, ccPtr, ccOwner;
    DevBuf itVal, itA, itPresent, itDiag, itIw, itVec;
    int itSys = 0;
    bool itUploaded = false;
};

// The full-batch step's CUDA graphs, kept across calls: a graph is replayed while every launch it holds would be the
// same (the key: the kernels' by-value arguments, the batch parts and the launch shapes), and captured again
// otherwise. Capture and instantiation of a step's ~1,400 launches is host work the device waits for.
struct StepGraphCache {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int64_t launches[2] = {0, 0};
    StepGraphCache() = default;
    StepGraphCache(const StepGraphCache&) = delete;
    StepGraphCache& operator=(const StepGraphCache&) = delete;
    ~StepGraphCache() { release(); }
    void release() {
        for (auto& x : exec)
            if (x) { cudaGraphExecDestroy(x); x = nullptr; }
        key.clear();
    }
};

}  // namespace gs

struct MatrixPattern;  // an analysed sparse-matrix pattern of the batched linear solve (kept per context)

struct gs_ctx {
    int device = 0;
    std::string lastError;
    std::mutex mu;
    cudaStream_t stream = nullptr;
    cudaStream_t partStream[2] = {nullptr, nullptr};  // part 1 of a batch's level sequences (part 0 runs on `stream`)
    int* pinnedCount = nullptr;
    std::map<std::string, int> multiTune;  // the multi-grid batch's CTA shape per set of grids (autotuned)
    std::vector<std::unique_ptr<MatrixPattern>> patterns;  // most recently used last
    unsigned long long* noallocScratch = nullptr;  // device address of the allocation-free check's static scratch
    bool clusterOk = false;  // the few-systems cluster walk can be scheduled on this device
    ~gs_ctx();
};

struct gs_grid {
    gs_ctx* ctx = nullptr;
    gs::HostGrid host;
    gs::Symbolic sym;
    std::vector<std::unique_ptr<gs::DevBuf>> bufs;
    gs::DevGrid view{};
    std::vector<double> pgen, qgen, pload, qload;
    gs::Workspace ws;
    gs::Workspace tws;  // compact copy of the few systems still stepping
    gs::Workspace mws;  // the full-batch step's systems still stepping, once many have converged (batch precision)
    std::unique_ptr<gs_grid> qgrid;  // the same grid analysed for Q-limit enforcement (built on first use)
    std::unique_ptr<gs_grid> rgrid;  // a twin with its own workspace for the DC-angle retries (built on first use)
    gs::OutageSetTable sets;         // multi-branch outages of the current call (view.nSet > 0 while installed)
    std::vector<gs::ElemSys> elemBatch;  // element outages of the systems in the workspace (empty: none)
    gs::DevBuf setBrBuf, setCellBuf, setRedBuf;
    int split = 0;      // first level run by the persistent kernels (factorisation)
    int splitB = 0;     // first level run by the persistent kernels in the triangular solves
    int tailSplit = 0;  // first level the few-systems path runs as one CTA per system
    int tailMax = gs::kTailMaxSystems;  // the few-systems path takes over at this many systems still stepping
    int psSplit = 0, psSplitB = 0;      // the same first persistent levels on the paired schedule
    bool paired = true;                 // the full-batch step and the cluster walk run the paired schedule
    // partial-pivoting mode (the re-solve of systems whose static pivot collapsed): every iteration steps on the
    // few-systems path with k_gp_solve in place of the static factorisation
    bool gpMode = false;
    gs::GpData gp;
    // the level-group cut and few-systems threshold in force (gs::SetSchedule; gs_screen_tune picks them)
    gs_schedule sched{2, 2, gs::kTailMaxSystems, 0, 0.0, 0.0, -1, {0, 0, 0}};
    gs::StepGraphCache stepGraphs[2];  // the full-batch step's graphs: [0] the whole batch, [1] the mid workspace
    // the subtree schedule of sched.subtree_cut (gs::BuildSubtrees) on the device; cut -1: none
    int subCut = -1, nSub = 0;
    gs::DevBuf subStage, subStagePtr, subWork;
};

struct MatrixPattern {
    uint64_t hash = 0;
    int n = 0;
    std::vector<int> rowPtr, colIdx, aSlot;
    std::unique_ptr<gs_grid> grid;  // the pattern's symbolic analysis, schedules and workspace (no Y, no buses)
    gs::DevBuf dSlot, dPinv;
};

gs_ctx::~gs_ctx() = default;

namespace gs {
namespace {

int SetErr(gs_ctx* c, int code, const std::string& msg) {
    if (c) { std::lock_guard<std::mutex> l(c->mu); c->lastError = msg; }
    return code;
}

#define GS_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) {                                                                        \
            int code_ = (e_ == cudaErrorMemoryAllocation) ? GS_ERR_OOM : GS_ERR_CUDA;                   \
            return SetErr(ctx, code_, std::string(#call) + ": " + cudaGetErrorString(e_));              \
        }                                                                                               \
    } while (0)

template <typename X>
int Upload(gs_grid* G, const std::vector<X>& v, const X** out) {
    gs_ctx* ctx = G->ctx;
    auto buf = std::make_unique<DevBuf>();
    GS_CUDA(buf->alloc(std::max<size_t>(sizeof(X), v.size() * sizeof(X))));
    if (!v.empty()) GS_CUDA(cudaMemcpy(buf->p, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice));
    *out = buf->as<X>();
    G->bufs.push_back(std::move(buf));
    return GS_OK;
}

// The grid's level-group cut and few-systems threshold. The persistent kernels take every level from the first
// one whose phases (and those of all levels above it) hold at most factorCut x kPersistWarps items (the
// factorisation, on the items of its two phases and of the backward substitution) or solveCut x kPersistWarps
// items (the triangular solves); the levels below run one launch per level and phase. The few-systems path takes
// over once at most tailMax systems still step.
void SetSchedule(gs_grid* G, const gs_schedule& sc) {
    const Symbolic& s = G->sym;
    G->sched = sc;
    G->tailMax = std::max(1, std::min(kTailMaxSystems, sc.tail_max));
    const int fCut = sc.factor_cut * kPersistWarps, sCut = sc.solve_cut * kPersistWarps;
    auto cuts = [&](const Symbolic::Schedule& f, const Symbolic::Schedule& b, const Symbolic::Schedule& v, int nLv,
                    int& split, int& splitB) {
        split = nLv;
        for (int l = nLv - 1; l >= 0; l--) {
            const auto& fp = f.levelItemPtr;
            const int a = fp[2 * l + 1] - fp[2 * l], bb = fp[2 * l + 2] - fp[2 * l + 1];
            const int c = b.levelItemPtr[l + 1] - b.levelItemPtr[l];
            if (std::max(std::max(a, bb), c) > fCut) break;
            split = l;
        }
        // the solves have one item per level for a few nodes (short pieces packed), so their persistent walk can
        // start lower in the tree than the factorisation's
        splitB = nLv;
        for (int l = nLv - 1; l >= 0; l--) {
            const int c = b.levelItemPtr[l + 1] - b.levelItemPtr[l];
            const int vv = v.levelItemPtr[l + 1] - v.levelItemPtr[l];
            if (std::max(c, vv) > sCut) break;
            splitB = l;
        }
        splitB = std::min(splitB, split);
    };
    cuts(s.factor, s.backward, s.forward, s.nLevels, G->split, G->splitB);
    if (s.ps.on) cuts(s.ps.factor, s.ps.backward, s.ps.forward, s.ps.nLevels, G->psSplit, G->psSplitB);
    // the subtrees below the subtree cut, kept below the persistent walk's first level
    const int cut = s.ps.on ? std::min(sc.subtree_cut, G->psSplit - 1) : -1;
    G->sched.subtree_cut = cut;
    if (cut != G->subCut) {
        G->subCut = -1;
        G->nSub = 0;
        if (cut >= 0) {
            const SubtreeSchedule st = BuildSubtrees(s, cut);
            auto up = [](DevBuf& d, const std::vector<int32_t>& h) {
                cudaError_t e = d.alloc(std::max<size_t>(1, h.size()) * 4);
                if (e == cudaSuccess && !h.empty()) e = cudaMemcpy(d.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
                return e;
            };
            if (st.nSub > 0 && up(G->subStage, st.subStage) == cudaSuccess &&
                up(G->subStagePtr, st.stagePtr) == cudaSuccess && up(G->subWork, st.work) == cudaSuccess) {
                G->subCut = cut;
                G->nSub = st.nSub;
            } else {
                cudaGetLastError();
                G->sched.subtree_cut = -1;  // no subtree schedule: every level its own launch
            }
        }
    }
}

// The subtree cut whose largest subtree holds at most `bytes` of FP32 LU for a system group (eight systems), or -1.
int SubtreeCutFor(const gs_grid* G, double bytes) {
    const Symbolic& s = G->sym;
    if (!s.ps.on) return -1;
    int best = -1;
    for (int cut = 0; cut < G->psSplit; cut++) {
        const SubtreeSchedule st = BuildSubtrees(s, cut);
        if ((double)st.maxEntries * 4.0 * 8.0 > bytes) break;
        best = cut;
    }
    return best;
}

int UploadGrid(gs_grid* G) {
    const HostGrid& h = G->host;
    const Symbolic& s = G->sym;
    DevGrid& v = G->view;
    v.n = s.n; v.m = s.m; v.nnzY = s.nnzY; v.nbr = s.nbr; v.nnzLU = s.nnzLU; v.nLevels = s.nLevels;
    v.qlim = s.qlim ? 1 : 0;
    v.qlimOn = v.qlim;
    v.qlimMaxPasses = kMaxQPasses;
    v.baseMva = h.base;
    const int n = h.n;
    G->pgen.assign(n, 0.0); G->qgen.assign(n, 0.0);
    for (int k = 0; k < h.ngen; k++) {
        if (!h.genOn[k]) continue;
        G->pgen[h.genBus[k]] += h.pg[k];
        G->qgen[h.genBus[k]] += h.qg[k];
    }
    G->pload.resize(n); G->qload.resize(n);
    for (int i = 0; i < n; i++) {
        G->pgen[i] /= h.base; G->qgen[i] /= h.base;
        G->pload[i] = h.pd[i] / h.base; G->qload[i] = h.qd[i] / h.base;
    }
    std::vector<double> rate(h.nbr), rateB(h.nbr), rateC(h.nbr);
    for (int k = 0; k < h.nbr; k++) {
        rate[k] = h.rateA[k] / h.base;
        rateB[k] = h.rateB[k] / h.base;
        rateC[k] = h.rateC[k] / h.base;
    }
    v.nBnd = h.nBnd;
    std::vector<int2> pairs(s.pairs.size() / 2);
    for (size_t q = 0; q < pairs.size(); q++) pairs[q] = make_int2(s.pairs[2 * q], s.pairs[2 * q + 1]);
    int rc;
#define UP(vec, field) if ((rc = Upload(G, vec, &v.field)) != GS_OK) return rc
    UP(s.yRowPtr, yRowPtr); UP(s.yCol, yCol); UP(s.yG, yG); UP(s.yB, yB);
    UP(s.brCell, brCell); UP(s.brRed, brRed); UP(s.brStamp, brStamp);
    UP(h.brF, brF); UP(h.brT, brT); UP(rate, rateA); UP(rateB, rateB); UP(rateC, rateC); UP(h.brOn, brOn);
    UP(h.bndPtr, bndPtr); UP(h.bndBranch, bndBranch); UP(h.bndDir, bndDir); UP(h.bndLimit, bndLimit);
    UP(G->pgen, pgen); UP(G->qgen, qgen); UP(G->pload, pload); UP(G->qload, qload);
    v.zip = nullptr;
    if (!h.zip.empty()) UP(h.zip, zip);
    {
        std::vector<double> qminPu(n), qmaxPu(n);
        for (int i = 0; i < n; i++) { qminPu[i] = s.qminMvar[i] / h.base; qmaxPu[i] = s.qmaxMvar[i] / h.base; }
        UP(qminPu, qminPu); UP(qmaxPu, qmaxPu); UP(s.qminMvar, qminMvar); UP(s.qmaxMvar, qmaxMvar);
    }
    UP(s.vm0, vm0); UP(s.va0, va0); UP(s.type0, busType); UP(s.busP, busP); UP(s.busQ, busQ); UP(s.ySlot, ySlot);
    UP(s.entSlot, entSlot); UP(s.entKind, entKind); UP(s.entHasA, entHasA);
    UP(s.entPairPtr, entPairPtr); UP(pairs, pairs); UP(s.diagPairNode, diagEnt); UP(s.levelNodes, levelNodes);
    UP(s.luBase, luBase); UP(s.luCnt, luCnt); UP(s.pRowPtr, pRowPtr); UP(s.pRows, pRows);
    UP(s.levelNodePtr, levelNodePtr); UP(s.entNode, entNode);
    {
        // work descriptors, one per schedule position
        auto entDesc = [&](int e) {
            return make_int4(s.entSlot[e], (int)s.entPairPtr[e], (int)s.entPairPtr[e + 1],
                             s.entKind[e] | (s.entHasA[e] << 2) | (s.entNode[e] << 3));
        };
        std::vector<int4> fd, vd, bd;
        for (int e : s.factor.work) fd.push_back(entDesc(e));
        for (int e : s.forward.work) vd.push_back(entDesc(e));
        for (int q : s.backward.work) {
            const int k = s.levelNodes[q];
            bd.push_back(make_int4(k, (int)s.luBase[k], s.luCnt[k], s.pRowPtr[k]));
        }
        UP(fd, fDesc); UP(vd, vDesc); UP(bd, bDesc);
    }
    UP(s.factor.work, fWork); UP(s.factor.items, fItems); UP(s.factor.levelItemPtr, fLevelPtr);
    UP(s.backward.work, bWork); UP(s.backward.items, bItems); UP(s.backward.levelItemPtr, bLevelPtr);
    UP(s.forward.work, vWork); UP(s.forward.items, vItems); UP(s.forward.levelItemPtr, vLevelPtr);
    UP(s.factor.levelWorkPtr, fWorkPtr); UP(s.backward.levelWorkPtr, bWorkPtr); UP(s.forward.levelWorkPtr, vWorkPtr);
    UP(s.factor.levelWide, fWide); UP(s.backward.levelWide, bWide); UP(s.forward.levelWide, vWide);
    UP(s.factor.levelMid, fMid); UP(s.backward.levelMid, bMid); UP(s.forward.levelMid, vMid);
    for (int w = 0; w < 2; w++) {
        const Symbolic::TopPart& t = s.top[w];
        DevTop& d = v.top[w];
        d.L0 = t.L0; d.nSlots = t.nSlots; d.nNodes = t.nNodes; d.nEnt = (int)t.ent.size();
        d.loadWide = t.loadWide; d.nLoad = (int)t.loadList.size();
        d.fwdLoadWide = t.fwdLoadWide; d.nFwdLoad = (int)t.fwdLoadList.size();
        std::vector<int2> ip(t.intPairs.size() / 2), ep(t.extPairs.size() / 2);
        for (size_t q = 0; q < ip.size(); q++) ip[q] = make_int2(t.intPairs[2 * q], t.intPairs[2 * q + 1]);
        for (size_t q = 0; q < ep.size(); q++) ep[q] = make_int2(t.extPairs[2 * q], t.extPairs[2 * q + 1]);
#define UPT(vec, field) if ((rc = Upload(G, vec, &d.field)) != GS_OK) return rc
        UPT(t.slotGlobal, slotGlobal); UPT(t.slotDiagNode, slotDiagNode); UPT(t.nodes, nodes); UPT(t.smemBase, smemBase);
        UPT(t.ent, ent); UPT(t.entSm, entSm); UPT(t.intPtr, intPtr); UPT(t.extPtr, extPtr);
        UPT(ip, intPairs); UPT(ep, extPairs); UPT(t.loadList, loadList); UPT(t.fwdLoadList, fwdLoadList);
        UPT(t.fWalk, fWalk); UPT(t.fWalkPtr, fWalkPtr); UPT(t.fWalkWide, fWalkWide);
        UPT(t.vWalk, vWalk); UPT(t.vWalkPtr, vWalkPtr); UPT(t.vWalkWide, vWalkWide);
        UPT(t.bWalk, bWalk); UPT(t.bWalkPtr, bWalkPtr); UPT(t.bWalkWide, bWalkWide);
        UPT(t.bRowPtr, bRowPtr); UPT(t.bRowSm, bRowSm);
#undef UPT
    }
    v.psLevels = 0;
    G->paired = std::getenv("GS_SCALAR_SCHEDULE") == nullptr;  // the scalar schedule everywhere, for comparison
    if (s.ps.on) {
        const Symbolic::PairSchedule& P = s.ps;
        std::vector<int2> pp(P.pairs.size() / 2);
        for (size_t q = 0; q < pp.size(); q++) pp[q] = make_int2(P.pairs[2 * q], P.pairs[2 * q + 1]);
        // descriptors in schedule order (position = work index)
        auto order = [](const std::vector<int32_t>& work, const std::vector<int32_t>& ta, const std::vector<int32_t>& tb,
                        std::vector<int4>& oa, std::vector<int4>& ob) {
            for (int t : work) {
                oa.push_back(make_int4(ta[4 * t], ta[4 * t + 1], ta[4 * t + 2], ta[4 * t + 3]));
                ob.push_back(make_int4(tb[4 * t], tb[4 * t + 1], tb[4 * t + 2], tb[4 * t + 3]));
            }
        };
        std::vector<int4> fa, fb, ba, bb, va, vb;
        order(P.factor.work, P.taskA, P.taskB, fa, fb);
        order(P.backward.work, P.bTaskA, P.bTaskB, ba, bb);
        order(P.forward.work, P.taskA, P.taskB, va, vb);
        UP(pp, psPairs);
        UP(fa, pfA); UP(fb, pfB); UP(ba, pbA); UP(bb, pbB); UP(va, pvA); UP(vb, pvB);
        UP(P.factor.items, pfItems); UP(P.backward.items, pbItems); UP(P.forward.items, pvItems);
        UP(P.factor.levelItemPtr, pfLevelPtr); UP(P.backward.levelItemPtr, pbLevelPtr); UP(P.forward.levelItemPtr, pvLevelPtr);
        UP(P.factor.levelWorkPtr, pfWorkPtr); UP(P.backward.levelWorkPtr, pbWorkPtr); UP(P.forward.levelWorkPtr, pvWorkPtr);
        UP(P.factor.levelWide, pfWide); UP(P.backward.levelWide, pbWide); UP(P.forward.levelWide, pvWide);
        UP(P.factor.levelMid, pfMid); UP(P.backward.levelMid, pbMid); UP(P.forward.levelMid, pvMid);
        v.psLevels = P.nLevels;
    }
#undef UP
    // the few-systems path runs the lowest levels as per-level launches while a phase of them holds more short
    // pieces than one CTA's threads (more than one round of a one-system walk)
    G->tailSplit = 0;
    for (int l = 0; l < s.nLevels; l++) {
        bool wideLevel = false;
        for (int ph = 0; ph < 2; ph++) {
            const int i = 2 * l + ph;
            if (s.factor.levelWorkPtr[i + 1] - s.factor.levelWorkPtr[i] - s.factor.levelWide[i] > kTailThreads) wideLevel = true;
        }
        if (s.backward.levelWorkPtr[l + 1] - s.backward.levelWorkPtr[l] - s.backward.levelWide[l] > kTailThreads) wideLevel = true;
        if (!wideLevel) break;
        G->tailSplit = l + 1;
    }
    SetSchedule(G, G->sched);
    return GS_OK;
}

size_t PerSystemBytes(const Symbolic& s, int precision) {
    size_t t = precision == GS_PREC_MIXED ? 4 : 8;
    size_t refine = precision == GS_PREC_MIXED ? (size_t)s.m * (t + 8) : 0;
    return (size_t)s.nnzLU * t + 2 * (size_t)s.m * t + refine + (size_t)s.n * 16 + (size_t)(s.nbr + s.n) * 9 + 256;
}

// classifyItems: items per system of the screen's classification (branches + boundaries + buses), 0 = none
int EnsureWs(gs_ctx* ctx, const Symbolic& s, Workspace& w, int B, int precision, int classifyItems, bool loadScale) {
    if (s.qlim) {
        const size_t nb = (size_t)s.n * B;
        GS_CUDA(w.effType.alloc(nb * 4)); GS_CUDA(w.qspecSys.alloc(nb * 8)); GS_CUDA(w.pinned.alloc(nb * 4));
        GS_CUDA(w.reverted.alloc(nb * 4)); GS_CUDA(w.qinj.alloc(nb * 8));
        GS_CUDA(w.passIter.alloc((size_t)B * 4)); GS_CUDA(w.qPass.alloc((size_t)B * 4)); GS_CUDA(w.qState.alloc((size_t)B * 4));
        GS_CUDA(w.ovBus.alloc((size_t)B * 8)); GS_CUDA(w.ovType.alloc((size_t)B * 8)); GS_CUDA(w.ovVm.alloc((size_t)B * 16));
        GS_CUDA(w.specBus.alloc((size_t)B * 4)); GS_CUDA(w.specDp.alloc((size_t)B * 8)); GS_CUDA(w.specDq.alloc((size_t)B * 8));
        GS_CUDA(w.specQmin.alloc((size_t)B * 8)); GS_CUDA(w.specQmax.alloc((size_t)B * 8));
    }
    size_t t = precision == GS_PREC_MIXED ? 4 : 8;
    size_t Bz = (size_t)B;
    GS_CUDA(w.vm.alloc(s.n * Bz * 8));
    GS_CUDA(w.va.alloc(s.n * Bz * 8));
    GS_CUDA(w.lu.alloc((size_t)s.nnzLU * Bz * t));
    GS_CUDA(w.y.alloc((size_t)s.m * Bz * t));
    GS_CUDA(w.piv.alloc((size_t)s.m * Bz * t));
    if (precision == GS_PREC_MIXED) {
        GS_CUDA(w.z.alloc((size_t)s.m * Bz * t));
        GS_CUDA(w.rhs64.alloc((size_t)s.m * Bz * 8));
        GS_CUDA(w.refine.alloc(Bz * 4));
    }
    GS_CUDA(w.maxMis.alloc(Bz * 8)); GS_CUDA(w.maxDx.alloc(Bz * 8));
    GS_CUDA(w.startMis.alloc(Bz * 8)); GS_CUDA(w.finalMis.alloc(Bz * 8)); GS_CUDA(w.beforeLast.alloc(Bz * 8));
    GS_CUDA(w.status.alloc(Bz * 4)); GS_CUDA(w.iters.alloc(Bz * 4)); GS_CUDA(w.active.alloc(Bz * 4));
    GS_CUDA(w.convIters.alloc(Bz * 4));
    GS_CUDA(w.flags.alloc(Bz * 4)); GS_CUDA(w.outage.alloc(Bz * 4)); GS_CUDA(w.activeCount.alloc(16));
    GS_CUDA(w.activeList.alloc(Bz * 4));
    GS_CUDA(w.origin.alloc(Bz * 4));
    GS_CUDA(w.startVm.alloc(s.n * 8)); GS_CUDA(w.startVa.alloc(s.n * 8));
    if (loadScale) GS_CUDA(w.loadScale.alloc(s.n * Bz * 8));
    if (classifyItems > 0) {
        const int nItems = classifyItems;
        GS_CUDA(w.code.alloc((size_t)nItems * Bz));
        GS_CUDA(w.value.alloc((size_t)nItems * Bz * 8));
        GS_CUDA(w.maxLoad.alloc(Bz * 8)); GS_CUDA(w.minVmNeg.alloc(Bz * 8)); GS_CUDA(w.maxVmB.alloc(Bz * 8));
        GS_CUDA(w.worstBnd.alloc(Bz * 8));
    }
    w.B = B;
    w.precision = precision;
    return GS_OK;
}

int EnsureWorkspace(gs_grid* G, int B, int precision, bool classify, bool loadScale) {
    // the compact workspace of the few-systems path (its interleave stride is set per compaction)
    const int cap = std::min(B, kCompactCap);
    // FP64 whatever the batch's precision: the few-systems path is latency-bound, so FP32 factors save nothing there
    // and would need the refinement solve
    (void)precision;
    int rc = EnsureWs(G->ctx, G->sym, G->tws, cap, GS_PREC_FP64, 0, loadScale);
    if (rc != GS_OK) return rc;
    return EnsureWs(G->ctx, G->sym, G->ws, B, precision, classify ? G->sym.nbr + G->host.nBnd + G->sym.n : 0,
                    loadScale);
}

// A batch view of workspace `w` with interleave stride B (at most the stride it was sized for).
DevBatch MakeBatchWs(const Workspace& w, int nLevels, int B, int count, bool useScale) {
    DevBatch b{};
    b.B = B; b.count = count;
    b.vm = w.vm.as<double>(); b.va = w.va.as<double>(); b.lu = w.lu.p; b.y = w.y.p; b.piv = w.piv.p;
    const bool mixed = w.precision == GS_PREC_MIXED;
    b.z = mixed ? w.z.p : nullptr;
    b.rhs64 = mixed ? w.rhs64.as<double>() : nullptr;
    b.refine = mixed ? w.refine.as<int>() : nullptr;
    b.maxMis = w.maxMis.as<unsigned long long>(); b.maxDx = w.maxDx.as<unsigned long long>();
    b.startMis = w.startMis.as<double>(); b.finalMis = w.finalMis.as<double>(); b.beforeLast = w.beforeLast.as<double>();
    b.status = w.status.as<int>(); b.iters = w.iters.as<int>(); b.active = w.active.as<int>();
    b.convIters = w.convIters.as<int>();
    b.flags = w.flags.as<int>(); b.outage = w.outage.as<int>();
    b.loadScale = useScale ? w.loadScale.as<double>() : nullptr;
    b.activeCount = w.activeCount.as<int>();
    b.activeList = w.activeList.as<int>();
    b.nLevels = nLevels;
    if (w.qState.p) {
        b.effType = w.effType.as<int>(); b.qspecSys = w.qspecSys.as<double>(); b.pinned = w.pinned.as<int>();
        b.reverted = w.reverted.as<int>(); b.qinj = w.qinj.as<double>(); b.passIter = w.passIter.as<int>();
        b.qPass = w.qPass.as<int>(); b.qState = w.qState.as<int>();
        if (w.ovOn) {
            b.ovBus = w.ovBus.as<int>(); b.ovType = w.ovType.as<int>(); b.ovVm = w.ovVm.as<double>();
            b.specBus = w.specBus.as<int>(); b.specDp = w.specDp.as<double>(); b.specDq = w.specDq.as<double>();
            b.specQmin = w.specQmin.as<double>(); b.specQmax = w.specQmax.as<double>();
        }
    }
    return b;
}

DevBatch MakeBatch(gs_grid* G, int count, bool useScale) {
    return MakeBatchWs(G->ws, G->sym.nLevels, G->ws.B, count, useScale);
}

// Parts of a full batch whose level sequences run side by side (parallel branches of the step graph).
constexpr int kParts = 2;  // measured on the 10,000-bus screen: 2 parts beat 1, 3 and 4 in mixed precision

// The systems [off, off + n) of batch b as a batch of their own (same interleave stride).
template <typename T>
DevBatch HalfView(const DevBatch& b, int off, int n) {
    DevBatch h = b;
    h.count = std::max(0, n);
    auto sh = [&](auto* p) { return p ? p + off : p; };
    h.vm = sh(b.vm); h.va = sh(b.va);
    h.lu = b.lu ? (void*)((T*)b.lu + off) : nullptr;
    h.piv = b.piv ? (void*)((T*)b.piv + off) : nullptr;
    h.y = b.y ? (void*)((T*)b.y + off) : nullptr;
    h.z = b.z ? (void*)((T*)b.z + off) : nullptr;
    h.rhs64 = sh(b.rhs64); h.refine = sh(b.refine); h.maxMis = sh(b.maxMis); h.maxDx = sh(b.maxDx);
    h.startMis = sh(b.startMis); h.finalMis = sh(b.finalMis); h.status = sh(b.status); h.iters = sh(b.iters);
    h.beforeLast = sh(b.beforeLast);
    h.convIters = sh(b.convIters); h.active = sh(b.active); h.flags = sh(b.flags); h.outage = sh(b.outage);
    h.loadScale = sh(b.loadScale);
    h.effType = sh(b.effType); h.qspecSys = sh(b.qspecSys); h.pinned = sh(b.pinned); h.reverted = sh(b.reverted);
    h.qinj = sh(b.qinj); h.passIter = sh(b.passIter); h.qPass = sh(b.qPass); h.qState = sh(b.qState);
    auto sh2 = [&](auto* p) { return p ? p + 2 * off : p; };  // two entries per system
    h.ovBus = sh2(b.ovBus); h.ovType = sh2(b.ovType); h.ovVm = sh2(b.ovVm);
    h.specBus = sh(b.specBus); h.specDp = sh(b.specDp); h.specDq = sh(b.specDq);
    h.specQmin = sh(b.specQmin); h.specQmax = sh(b.specQmax);
    return h;
}

// Run the Newton iteration of `count` systems already placed in the workspace (outage, loadScale).
// `startFromWs`: start every system from ws.startVm / startVa (a solved base), else from the grid start.
// The partial-pivoting re-solve's marks: a solved system is flagged kFlagPivoted; one the factorisation could not
// solve (singular at the row floor, out of capacity, not finite) has its step refused (its run stops with the state
// it has, as NewtonShell.SolveStep's refusal stops the reference's) and is flagged kFlagPivotFailed.
__global__ void k_gp_mark(DevBatch b, const int* list, const int* result, int nList) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nList) return;
    const int s = list[q];
    if (result[q] == GP_OK || result[q] == GP_ITERATIVE) atomicOr(&b.flags[s], kFlagPivoted);
    else atomicOr(&b.flags[s], kFlagPivotFailed | kFlagStepBad);
}

// The step of the listed systems of batch `cur` (FP64; Jacobian or matrix in its LU slots, right-hand side in y, both
// before any static factorisation) by the partial-pivoting factorisation, in chunks the scratch holds; the solution
// replaces y. Returns the kernels launched.
int GpStep(gs_grid* G, const DevBatch& cur, const int* dList, int nList, cudaStream_t st, int* launched,
           bool iterative = false, double tol = 1e-8) {
    gs_ctx* ctx = G->ctx;
    const Symbolic& s = G->sym;
    GpData& d = G->gp;
    *launched = 0;
    if (nList <= 0) return GS_OK;
    const int m = s.m;
    if (!d.uploaded) {
        GS_CUDA(d.colPtr.alloc((s.aColPtr.size()) * 4));
        GS_CUDA(d.row.alloc(std::max<size_t>(1, s.aRow.size()) * 4));
        GS_CUDA(d.slot.alloc(std::max<size_t>(1, s.aSlot.size()) * 4));
        GS_CUDA(cudaMemcpy(d.colPtr.p, s.aColPtr.data(), s.aColPtr.size() * 4, cudaMemcpyHostToDevice));
        if (!s.aRow.empty()) {
            GS_CUDA(cudaMemcpy(d.row.p, s.aRow.data(), s.aRow.size() * 4, cudaMemcpyHostToDevice));
            GS_CUDA(cudaMemcpy(d.slot.p, s.aSlot.data(), s.aSlot.size() * 4, cudaMemcpyHostToDevice));
        }
        d.uploaded = true;
    }
    // L and U capacity per system: twice the static pattern's entries, plus room for rows pivoted off the diagonal
    const int64_t cap = 2 * s.nnzLU + 8 * (int64_t)m;
    const size_t perSys = (size_t)m * (8 + 8 + 4 * 4) + 2 * (size_t)(m + 1) * 4 + (size_t)cap * 24 + 4;
    // systems per launch: up to two per SM, within 2 GB of scratch
    const int want = (int)std::max<size_t>(1, std::min<size_t>(296, ((size_t)2 << 30) / perSys));
    if (d.maxSys < want || d.cap != cap) {
        const size_t k = (size_t)want;
        GS_CUDA(d.x.alloc(k * m * 8)); GS_CUDA(d.rowMax.alloc(k * m * 8));
        GS_CUDA(d.xi.alloc(k * m * 4)); GS_CUDA(d.pstack.alloc(k * m * 4)); GS_CUDA(d.mark.alloc(k * m * 4));
        GS_CUDA(d.pinv.alloc(k * m * 4));
        GS_CUDA(d.lp.alloc(k * (m + 1) * 4)); GS_CUDA(d.up.alloc(k * (m + 1) * 4));
        GS_CUDA(d.li.alloc(k * cap * 4)); GS_CUDA(d.ui.alloc(k * cap * 4));
        GS_CUDA(d.lx.alloc(k * cap * 8)); GS_CUDA(d.ux.alloc(k * cap * 8));
        GS_CUDA(d.result.alloc(k * 4));
        d.maxSys = want;
        d.cap = cap;
    }
    GpView v{};
    v.m = m; v.cap = cap;
    v.colPtr = d.colPtr.as<int>(); v.row = d.row.as<int>(); v.slot = d.slot.as<int>();
    v.x = d.x.as<double>(); v.rowMax = d.rowMax.as<unsigned long long>();
    v.xi = d.xi.as<int>(); v.pstack = d.pstack.as<int>(); v.mark = d.mark.as<int>(); v.pinv = d.pinv.as<int>();
    v.lp = d.lp.as<int>(); v.up = d.up.as<int>(); v.li = d.li.as<int>(); v.ui = d.ui.as<int>();
    v.lx = d.lx.as<double>(); v.ux = d.ux.as<double>(); v.result = d.result.as<int>();
    IterView iv{};
    if (iterative) {
        // NewtonShell.SolveStep's fallback when the factorisation finds the Jacobian singular (NewtonShell.cs:96-105)
        if (!d.itUploaded) {
            auto up = [&](DevBuf& buf, const std::vector<int>& h) -> cudaError_t {
                cudaError_t e = buf.alloc(std::max<size_t>(1, h.size()) * 4);
                if (e == cudaSuccess && !h.empty()) e = cudaMemcpy(buf.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice);
                return e;
            };
            GS_CUDA(up(d.jRowPtr, s.jRowPtr)); GS_CUDA(up(d.jCol, s.jCol)); GS_CUDA(up(d.jSlot, s.jSlot));
            GS_CUDA(up(d.jYcell, s.jYcell)); GS_CUDA(up(d.eqPinv, s.pinv)); GS_CUDA(up(d.ccPtr, s.ccPtr));
            GS_CUDA(up(d.ccOwner, s.ccOwner));
            d.itUploaded = true;
        }
        if (d.itSys < d.maxSys) {
            const size_t k = (size_t)d.maxSys, nz = (size_t)std::max(1, s.nnzJ);
            GS_CUDA(d.itVal.alloc(k * nz * 8)); GS_CUDA(d.itA.alloc(k * nz * 8)); GS_CUDA(d.itPresent.alloc(k * nz * 4));
            GS_CUDA(d.itDiag.alloc(k * m * 4)); GS_CUDA(d.itIw.alloc(k * m * 4)); GS_CUDA(d.itVec.alloc(k * 10 * m * 8));
            d.itSys = d.maxSys;
        }
        iv.m = m; iv.nnz = s.nnzJ; iv.nbr = s.nbr;
        iv.rowPtr = d.jRowPtr.as<int>(); iv.col = d.jCol.as<int>(); iv.slot = d.jSlot.as<int>();
        iv.ycell = d.jYcell.as<int>(); iv.pinv = d.eqPinv.as<int>(); iv.ccPtr = d.ccPtr.as<int>();
        iv.ccOwner = d.ccOwner.as<int>(); iv.setBr = G->view.setBr; iv.outage = cur.outage;
        iv.tol = std::min(1e-10, tol * 1e-3);  // NumericTolerances.cs:256-260
        iv.maxIter = 4 * m + 200;
        iv.budgetNs = 2000000000LL;  // a run that has not converged in 2 s gives up (GP_TIMEOUT)
        iv.val = d.itVal.as<double>(); iv.a = d.itA.as<double>(); iv.present = d.itPresent.as<int>();
        iv.diag = d.itDiag.as<int>(); iv.iw = d.itIw.as<int>(); iv.vec = d.itVec.as<double>(); iv.result = v.result;
    }
    for (int off = 0; off < nList; off += d.maxSys) {
        const int c = std::min(d.maxSys, nList - off);
        k_gp_solve<<<c, 32, 0, st>>>(v, (const double*)cur.lu, (double*)cur.y, cur.B, dList + off, c);
        if (iterative) {
            k_gp_iterative<<<c, 32, 0, st>>>(iv, (const double*)cur.lu, (double*)cur.y, cur.B, dList + off, c, s.nbr);
            *launched += 1;
        }
        k_gp_mark<<<(c + 127) / 128, 128, 0, st>>>(cur, dList + off, v.result, c);
        *launched += 2;
    }
    GS_CUDA(cudaGetLastError());
    return GS_OK;
}

struct NewtonStats {
    int64_t launches = 0;
    int iterations = 0;
    double factorMs = 0, solveMs = 0, mismatchMs = 0, otherMs = 0;
    double factorBytes = 0;
    double levelFactorMs = 0, levelFactorBytes = 0, tailMs = 0;
};

template <typename T>
int Newton(gs_grid* G, int count, bool useScale, bool startFromWs, const gs_pf_opts& o, float* ms,
           NewtonStats* stats = nullptr, const double* vmSys = nullptr, const double* vaSys = nullptr) {
    gs_ctx* ctx = G->ctx;
    const Symbolic& s = G->sym;
    Workspace& w = G->ws;
    cudaStream_t st = ctx->stream;
    DevBatch b = MakeBatch(G, count, useScale);
    const DevGrid& g = G->view;
    const int groups = w.B / 32;
    cudaEvent_t e0, e1;
    GS_CUDA(cudaEventCreate(&e0));
    GS_CUDA(cudaEventCreate(&e1));
    GS_CUDA(cudaEventRecord(e0, st));
    dim3 blk8(32, 8), blk4(32, 4);
    k_init<<<dim3((s.n + 7) / 8, groups), blk8, 0, st>>>(g, b, startFromWs ? w.startVm.as<double>() : nullptr,
                                                          startFromWs ? w.startVa.as<double>() : nullptr, vmSys, vaSys);
    GS_CUDA(cudaGetLastError());
    // the step (factor levels, backward levels, refinement, max |dx|, update) as one graph
    const int refine = sizeof(T) < sizeof(double) ? 1 : 0;
    const bool timed = o.phase_timing != 0;
    cudaEvent_t ev[5];
    if (timed) for (auto& e : ev) GS_CUDA(cudaEventCreate(&e));
    int64_t stepLaunches = 0;
    // levels [0, split) run one launch per level (wide: thousands of tasks); levels [split, nLevels) run in
    // one persistent launch per phase (narrow: a few tasks per level, latency-bound)
    // the full-batch step runs the paired schedule (units of one node or a 2 x 2 pair) where the grid has one
    const bool pairedOn = G->paired && g.psLevels > 0;
    const int nLv = pairedOn ? g.psLevels : s.nLevels;
    const int split = pairedOn ? G->psSplit : G->split, splitB = pairedOn ? G->psSplitB : G->splitB;
    const int persistThreads = 32;
    // warps per persistent CTA: as many as let every system group's CTA be resident at once (one wave), at most
    // kPersistWarps (a second partial wave would double the launch)
    // The batch the full-batch step runs on: the whole batch, or (after a compaction) its systems still stepping in
    // the mid workspace. Its parts run their level sequences as parallel branches of the step's graph, so that one
    // part's dependent-load latency and wave tails overlap the other's; small batches run as one. parts: as many as
    // keep each part at 148 or more system groups and at least one system, at most kParts.
    DevBatch stepB = b;
    int persistWarps[3] = {kPersistWarps, kPersistWarps, kPersistWarps};  // per walk: factorisation, backward, forward
    int parts = 1;
    DevBatch hb[kParts];
    auto setParts = [&](const DevBatch& base) {
        // warps per persistent CTA, for each walk (the three kernels use different numbers of registers): as many as
        // let every system group's CTA be resident at once (one wave), at most kPersistWarps. A second wave doubles
        // the walk: measured on the 10,000-bus screen, the backward walk (104 registers a thread) sized by the
        // factorisation's (90) ran 625 CTAs in two waves of 592.
        int sms = 0, occ = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
        const void* pks[3] = {
            pairedOn ? (const void*)k_ppersistent<T, kWorkFactor> : (const void*)k_persistent<T, kWorkFactor>,
            pairedOn ? (const void*)k_ppersistent<T, kWorkBackward> : (const void*)k_persistent<T, kWorkBackward>,
            pairedOn ? (const void*)k_ppersistent<T, kWorkForward> : (const void*)k_persistent<T, kWorkForward>};
        for (int wk = 0; wk < 3; wk++)
            for (int wpc = kPersistWarps; wpc >= 1; wpc--) {
                persistWarps[wk] = wpc;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, pks[wk], 32 * wpc, 0) == cudaSuccess &&
                    (int64_t)occ * sms >= base.B / Lay<T>::S)
                    break;
            }
        const int cnt = base.count;
        parts = 1;
        const int groupsAll = base.B / Lay<T>::S;
        while (parts < kParts && groupsAll / (parts + 1) >= 148 && cnt > (base.B / (parts + 1)) * parts) parts++;
        const int per = (base.B / parts) / 32 * 32;
        for (int q = 0; q < parts; q++) {
            const int off = q * per, n = q == parts - 1 ? cnt - off : std::min(per, cnt - off);
            hb[q] = q == 0 ? base : HalfView<T>(base, off, n);
            if (q == 0) hb[0].count = std::min(cnt, parts == 1 ? cnt : per);
        }
    };
    setParts(b);
    cudaEvent_t evFork, evJoin[kParts];
    GS_CUDA(cudaEventCreateWithFlags(&evFork, cudaEventDisableTiming));
    for (auto& e : evJoin) GS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    auto launchLevel = [&](const DevBatch& bb, cudaStream_t ss, auto kernel, T* vec, int i0, int i1) {
        const int grp = (bb.count + Lay<T>::S - 1) / Lay<T>::S;
        if (i1 > i0 && grp > 0) { kernel<<<dim3((i1 - i0 + 3) / 4, grp), blk4, 0, ss>>>(g, bb, vec, i0, i1); stepLaunches++; }
    };
    const auto& fp = pairedOn ? s.ps.factor.levelItemPtr : s.factor.levelItemPtr;
    const auto& bp = pairedOn ? s.ps.backward.levelItemPtr : s.backward.levelItemPtr;
    const auto& vp = pairedOn ? s.ps.forward.levelItemPtr : s.forward.levelItemPtr;
    // one level of schedule W: the paired kernels or the scalar ones
    auto level = [&](const DevBatch& bb, cudaStream_t ss, auto wTag, T* vec, int i0, int i1) {
        constexpr int W = decltype(wTag)::value;
        if (pairedOn) launchLevel(bb, ss, k_plevel<T, W>, vec, i0, i1);
        else launchLevel(bb, ss, k_level<T, W>, vec, i0, i1);
    };
    auto persistent = [&](const DevBatch& bb, cudaStream_t ss, auto wTag, T* vec, int l0) {
        constexpr int W = decltype(wTag)::value;
        const int wk = W == kWorkFactor ? 0 : (W == kWorkBackward ? 1 : 2);
        const dim3 grid((bb.count + Lay<T>::S - 1) / Lay<T>::S), blk(persistThreads, persistWarps[wk]);
        if (pairedOn) k_ppersistent<T, W><<<grid, blk, 0, ss>>>(g, bb, vec, l0, nLv);
        else k_persistent<T, W><<<grid, blk, 0, ss>>>(g, bb, vec, l0, nLv);
        stepLaunches++;
    };
    using FW = std::integral_constant<int, kWorkFactor>;
    using BW = std::integral_constant<int, kWorkBackward>;
    using VW = std::integral_constant<int, kWorkForward>;
    auto factorPhase = [&](const DevBatch& bb, cudaStream_t ss) {
        int l0 = 0;
        if (pairedOn && G->subCut >= 0 && G->nSub > 0) {  // the subtrees below the cut: one launch
            const int grp = (bb.count + Lay<T>::S - 1) / Lay<T>::S;
            if (grp > 0) {
                k_psubtree<T><<<dim3(grp, G->nSub), blk4, 0, ss>>>(g, bb, G->subStage.as<int>(), G->subStagePtr.as<int>(),
                                                                 G->subWork.as<int>());
                stepLaunches++;
            }
            l0 = G->subCut + 1;
        }
        for (int l = l0; l < split; l++) {
            level(bb, ss, FW{}, (T*)bb.y, fp[2 * l], fp[2 * l + 1]);
            level(bb, ss, FW{}, (T*)bb.y, fp[2 * l + 1], fp[2 * l + 2]);
        }
        if (split < nLv) persistent(bb, ss, FW{}, (T*)bb.y, split);
    };
    auto backward = [&](const DevBatch& bb, cudaStream_t ss, T* vec) {
        if (splitB < nLv) persistent(bb, ss, BW{}, vec, splitB);
        for (int l = splitB - 1; l >= 0; l--) level(bb, ss, BW{}, vec, bp[l], bp[l + 1]);
    };
    auto solvePhase = [&](const DevBatch& bb, cudaStream_t ss, bool doRefine) {
        backward(bb, ss, (T*)bb.y);
        if (doRefine) {
            k_residual<T><<<dim3((s.n + 7) / 8, (bb.count + 31) / 32), blk8, 0, ss>>>(g, bb, nullptr, 0);
            stepLaunches++;
            for (int l = 0; l < splitB; l++) level(bb, ss, VW{}, (T*)bb.z, vp[l], vp[l + 1]);
            if (splitB < nLv) persistent(bb, ss, VW{}, (T*)bb.z, splitB);
            backward(bb, ss, (T*)bb.z);
        }
    };
    // a phase over every part: parts 1.. on their own streams, forked from and joined back into st
    auto bothHalves = [&](auto&& phase) {
        if (parts == 1) { phase(hb[0], st); return; }
        cudaEventRecord(evFork, st);
        for (int q = 1; q < parts; q++) {
            cudaStreamWaitEvent(ctx->partStream[q], evFork, 0);
            phase(hb[q], ctx->partStream[q]);
        }
        phase(hb[0], st);
        for (int q = 1; q < parts; q++) {
            cudaEventRecord(evJoin[q], ctx->partStream[q]);
            cudaStreamWaitEvent(st, evJoin[q], 0);
        }
    };
    const int rowsPerBlock = 512;
    auto updatePhase = [&](bool doRefine) {
        const int grp = stepB.B / 32;
        k_dxmax<T><<<dim3((s.m + rowsPerBlock - 1) / rowsPerBlock, grp), blk8, 0, st>>>(g, stepB, rowsPerBlock, doRefine, nullptr, 0);
        k_update<T><<<dim3((s.n + 7) / 8, grp), blk8, 0, st>>>(g, stepB, doRefine, nullptr, 0);
        stepLaunches += 2;
    };
    // The full-batch step as a graph; mixed precision keeps a second graph with the refinement solve, launched
    // only in iterations where some system refines (k_status counts them).
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int64_t launchesPerStep[2] = {0, 0};
    cudaError_t ce = cudaSuccess;
    // (re)capture the step graphs for stepB (its parts set)
    auto captureStep = [&]() -> int {
        exec[0] = exec[1] = nullptr;
        if (timed || G->gpMode) return GS_OK;  // the partial-pivoting re-solve never takes a full-batch step
        // the graphs of the last call on this workspace are replayed when they hold the same launches
        StepGraphCache& gc = G->stepGraphs[stepB.lu == b.lu ? 0 : 1];
        std::vector<unsigned char> key;
        auto put = [&](const void* p, size_t n) {
            const unsigned char* c = static_cast<const unsigned char*>(p);
            key.insert(key.end(), c, c + n);
        };
        const int shape[12] = {(int)sizeof(T), refine, parts, persistWarps[0], persistWarps[1], persistWarps[2], split,
                               splitB, pairedOn ? 1 : 0, nLv, G->subCut, G->nSub};
        put(shape, sizeof shape);
        const void* subPtrs[3] = {G->subStage.p, G->subStagePtr.p, G->subWork.p};
        put(subPtrs, sizeof subPtrs);
        put(&g, sizeof g);
        put(&stepB, sizeof stepB);
        for (int q = 0; q < parts; q++) put(&hb[q], sizeof hb[q]);
        if (gc.exec[0] && gc.key == key) {
            for (int r = 0; r <= refine; r++) { exec[r] = gc.exec[r]; launchesPerStep[r] = gc.launches[r]; }
            return GS_OK;
        }
        gc.release();
        for (int r = 0; r <= refine; r++) {
            cudaGraph_t graph;
            stepLaunches = 0;
            GS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            bothHalves([&](const DevBatch& bb, cudaStream_t ss) {
                factorPhase(bb, ss);
                solvePhase(bb, ss, r != 0);
            });
            updatePhase(r != 0);
            ce = cudaStreamEndCapture(st, &graph);
            if (ce == cudaSuccess) {
                ce = cudaGraphInstantiate(&gc.exec[r], graph, 0);
                cudaGraphDestroy(graph);
            }
            if (ce != cudaSuccess) {
                gc.release();
                return SetErr(ctx, GS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
            }
            gc.launches[r] = launchesPerStep[r] = stepLaunches;
            exec[r] = gc.exec[r];
        }
        gc.key = std::move(key);
        return GS_OK;
    };
    if (int rcCap = captureStep(); rcCap != GS_OK) {
        cudaEventDestroy(evFork);
        for (auto& e : evJoin) cudaEventDestroy(e);
        return rcCap;
    }
    const char* traceEnv = std::getenv("GS_TRACE_ITERATIONS");  // per-iteration phase times (with phase_timing)
    const bool traceIters = traceEnv && traceEnv[0] == '1';
    int64_t launches = 1;
    int iterations = 0;
    int64_t sysIters = 0;  // systems stepped, summed over the iterations
    int64_t levelSys = 0;  // the same over full-batch iterations
    double fMs = 0, sMs = 0, mMs = 0, oMs = 0, lfMs = 0, tMs = 0;
    int rc = GS_OK;
    int listCount = 0;  // > 0: cur.activeList holds the systems of the previous few-systems iteration
    // The batch being stepped: the full one, or (few-systems path) a compact copy of its last systems.
    DevBatch cur = b;
    bool compacted = false;
    bool midOn = false;  // cur is the mid workspace (its origin list maps it back to b)
    const dim3 nodeBlocks((s.n + 7) / 8);
    // with Q limits every pass may take up to max_iterations steps (plus the step-less pass switches)
    const int maxLoop = g.qlim ? (o.max_iterations + 2) * (g.qlimMaxPasses + 2) : o.max_iterations + 4;
    for (int iter = 0; iter <= maxLoop; iter++) {
        if (timed) cudaEventRecord(ev[0], st);
        if (listCount > 0)
            k_mismatch_jac<double><<<dim3(nodeBlocks.x, (listCount + 31) / 32), blk8, 0, st>>>(g, cur, 1, nullptr, nullptr,
                                                                                       cur.activeList, listCount);
        else
            k_mismatch_jac<T><<<dim3(nodeBlocks.x, cur.B / 32), blk8, 0, st>>>(g, cur, 1, nullptr, nullptr, nullptr, 0);
        if (timed) cudaEventRecord(ev[1], st);
        cudaMemsetAsync(cur.activeCount, 0, 2 * sizeof(int), st);
        if (g.qlim) {
            k_status_q<<<(cur.count + 255) / 256, 256, 0, st>>>(cur, o.tolerance, o.diverge_limit_pu, o.max_iterations);
            k_qapply<<<dim3(nodeBlocks.x, cur.B / 32), blk8, 0, st>>>(g, cur);
            k_qrevert<<<dim3(nodeBlocks.x, cur.B / 32), blk8, 0, st>>>(g, cur);
            k_qfinish<<<(cur.count + 255) / 256, 256, 0, st>>>(cur, g.qlimMaxPasses);
            launches += 3;
        } else {
            k_status<<<(cur.count + 255) / 256, 256, 0, st>>>(cur, iter, o.tolerance, o.diverge_limit_pu, o.max_iterations);
        }
        launches += 2;
        cudaMemcpyAsync(ctx->pinnedCount, cur.activeCount, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
        ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) { rc = SetErr(ctx, GS_ERR_CUDA, std::string("newton: ") + cudaGetErrorString(ce)); break; }
        if (timed) { float t; cudaEventElapsedTime(&t, ev[0], ev[1]); mMs += t; }
        if (*ctx->pinnedCount == 0) break;
        iterations++;
        const int nActive = ctx->pinnedCount[0];
        const int anyRefine = refine && ctx->pinnedCount[1] > 0 ? 1 : 0;
        sysIters += nActive;
        if (nActive <= G->tailMax || G->gpMode) {
            if (midOn) {  // the mid workspace's systems go back to the batch, which the few-systems path gathers from
                k_scatter<<<dim3(nodeBlocks.x, cur.B / 32), blk8, 0, st>>>(cur, b, G->mws.origin.as<int>(), s.n);
                launches++;
                cur = b;
                midOn = false;
            }
            if (timed) cudaEventRecord(ev[1], st);
            const int stride = (nActive + 31) / 32 * 32;
            if (!compacted || 2 * stride <= cur.B) {
                // (re)compact: the full batch takes back the compact systems, then the active ones move out
                if (compacted) {
                    k_scatter<<<dim3(nodeBlocks.x, cur.B / 32), blk8, 0, st>>>(cur, b, G->tws.origin.as<int>(), s.n);
                    launches++;
                }
                cudaMemsetAsync(b.activeCount, 0, sizeof(int), st);
                k_collect_active<<<(count + 255) / 256, 256, 0, st>>>(b);
                cudaMemcpyAsync(G->tws.origin.p, b.activeList, nActive * sizeof(int), cudaMemcpyDeviceToDevice, st);
                cur = MakeBatchWs(G->tws, s.nLevels, stride, nActive, useScale);
                k_gather<<<dim3(nodeBlocks.x, stride / 32), blk8, 0, st>>>(b, cur, G->tws.origin.as<int>(), s.n);
                // this iteration's Jacobian and right-hand side, rebuilt in the compact workspace; the mismatch
                // maximum it records was already taken by k_status
                k_mismatch_jac<double><<<dim3(nodeBlocks.x, stride / 32), blk8, 0, st>>>(g, cur, 1, nullptr, nullptr, nullptr, 0);
                cudaMemsetAsync(cur.maxMis, 0, (size_t)nActive * sizeof(unsigned long long), st);
                launches += 3;
                compacted = true;
            }
            // few systems left: the wide bottom levels as per-level launches over the compact batch, the rest as
            // one CTA per active system (k_tail), in FP64 (the compact workspace's precision)
            cudaMemsetAsync(cur.activeCount, 0, sizeof(int), st);
            k_collect_active<<<(cur.count + 255) / 256, 256, 0, st>>>(cur);
            if (G->gpMode) {
                // the partial-pivoting re-solve: the step by k_gp_solve from the Jacobian just filled
                if (timed) cudaEventRecord(ev[2], st);
                int gl = 0;
                if ((rc = GpStep(G, cur, cur.activeList, nActive, st, &gl, true, o.tolerance)) != GS_OK) break;
                launches += 1 + gl;
            } else {
                launches += 1 + FewSystemsSolve<double>(g, cur, s, nActive, G->tailSplit, false, st,
                                                        timed ? ev[2] : nullptr, ctx->clusterOk, G->paired);
            }
            if (timed) cudaEventRecord(ev[3], st);
            {
                const int grp = (nActive + 31) / 32;
                k_dxmax<double><<<dim3((s.m + rowsPerBlock - 1) / rowsPerBlock, grp), blk8, 0, st>>>(g, cur, rowsPerBlock, 0,
                                                                                               cur.activeList, nActive);
                k_update<double><<<dim3(nodeBlocks.x, grp), blk8, 0, st>>>(g, cur, 0, cur.activeList, nActive);
                launches += 2;
            }
            listCount = nActive;
            if (timed) {
                cudaEventRecord(ev[4], st);
                ce = cudaEventSynchronize(ev[4]);
                if (ce != cudaSuccess) { rc = SetErr(ctx, GS_ERR_CUDA, std::string("newton: ") + cudaGetErrorString(ce)); break; }
                float t1, t2, t3;
                cudaEventElapsedTime(&t1, ev[1], ev[2]);
                cudaEventElapsedTime(&t2, ev[2], ev[3]);
                cudaEventElapsedTime(&t3, ev[3], ev[4]);
                fMs += t1; sMs += t2; oMs += t3; tMs += t1 + t2 + t3;
                if (traceIters)
                    std::fprintf(stderr, "gs: iteration %d active %d (few-systems path) factor %.3f ms solve %.3f ms update %.3f ms\n",
                                 iter, nActive, t1, t2, t3);
            }
            continue;
        }
        // Many systems converged but more than the few-systems path takes: the ones still stepping move into the mid
        // workspace (same precision, stride their count rounded up to 32) and the step graph is captured for it, so
        // the converged systems' warps are not launched again. Measured on the 10,000-bus screen: the third iteration
        // (2,998 of 5,000 stepping) cost as much as the first before this.
        if (nActive < kMidCompactBelow * cur.count && !std::getenv("GS_NO_MID_COMPACT")) {
            const int B2 = (nActive + 31) / 32 * 32;
            G->mws.ovOn = w.ovOn;
            if (EnsureWs(ctx, s, G->mws, std::max(B2, G->mws.B), w.precision, 0, useScale) == GS_OK) {
                if (midOn) {
                    k_scatter<<<dim3(nodeBlocks.x, cur.B / 32), blk8, 0, st>>>(cur, b, G->mws.origin.as<int>(), s.n);
                    launches++;
                }
                cudaMemsetAsync(b.activeCount, 0, sizeof(int), st);
                k_collect_active<<<(count + 255) / 256, 256, 0, st>>>(b);
                cudaMemcpyAsync(G->mws.origin.p, b.activeList, nActive * sizeof(int), cudaMemcpyDeviceToDevice, st);
                const DevBatch mid = MakeBatchWs(G->mws, s.nLevels, B2, nActive, useScale);
                k_gather<<<dim3(nodeBlocks.x, B2 / 32), blk8, 0, st>>>(b, mid, G->mws.origin.as<int>(), s.n);
                // this iteration's Jacobian and right-hand side, rebuilt in the mid workspace; the mismatch maximum it
                // records was already taken by k_status
                k_mismatch_jac<T><<<dim3(nodeBlocks.x, B2 / 32), blk8, 0, st>>>(g, mid, 1, nullptr, nullptr, nullptr, 0);
                cudaMemsetAsync(mid.maxMis, 0, (size_t)nActive * sizeof(unsigned long long), st);
                launches += 3;
                cur = mid;
                stepB = mid;
                midOn = true;
                setParts(mid);
                if ((rc = captureStep()) != GS_OK) break;
            } else {
                cudaGetLastError();  // no room for the mid workspace: keep stepping the whole batch
            }
        }
        if (!timed) {
            ce = cudaGraphLaunch(exec[anyRefine], st);
            launches += launchesPerStep[anyRefine];
            if (ce != cudaSuccess) { rc = SetErr(ctx, GS_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(ce)); break; }
        } else {
            stepLaunches = 0;
            cudaEventRecord(ev[1], st);
            bothHalves([&](const DevBatch& bb, cudaStream_t ss) { factorPhase(bb, ss); });
            cudaEventRecord(ev[2], st);
            bothHalves([&](const DevBatch& bb, cudaStream_t ss) { solvePhase(bb, ss, anyRefine != 0); });
            cudaEventRecord(ev[3], st);
            updatePhase(anyRefine != 0);
            cudaEventRecord(ev[4], st);
            launches += stepLaunches;
            ce = cudaEventSynchronize(ev[4]);
            if (ce != cudaSuccess) { rc = SetErr(ctx, GS_ERR_CUDA, std::string("newton: ") + cudaGetErrorString(ce)); break; }
            float t1, t2, t3;
            cudaEventElapsedTime(&t1, ev[1], ev[2]);
            cudaEventElapsedTime(&t2, ev[2], ev[3]);
            cudaEventElapsedTime(&t3, ev[3], ev[4]);
            fMs += t1; sMs += t2; oMs += t3; lfMs += t1;
            levelSys += nActive;
            if (traceIters)
                std::fprintf(stderr, "gs: iteration %d active %d factor %.3f ms solve %.3f ms update %.3f ms\n", iter,
                             *ctx->pinnedCount, t1, t2, t3);
        }
    }
    if (compacted && rc == GS_OK) {
        k_scatter<<<dim3(nodeBlocks.x, cur.B / 32), blk8, 0, st>>>(cur, b, G->tws.origin.as<int>(), s.n);
        launches++;
    } else if (midOn && rc == GS_OK) {
        k_scatter<<<dim3(nodeBlocks.x, cur.B / 32), blk8, 0, st>>>(cur, b, G->mws.origin.as<int>(), s.n);
        launches++;
    }
    if (timed) for (auto& e : ev) cudaEventDestroy(e);
    if (stats) {
        stats->launches += launches;
        stats->iterations = std::max(stats->iterations, iterations);
        stats->factorMs += fMs; stats->solveMs += sMs; stats->mismatchMs += mMs; stats->otherMs += oMs;
        // algorithmic bytes of one factorisation per system: read J (nnzJ) + write L and U (nnzLU)
        stats->factorBytes += (double)sysIters * (double)sizeof(T) * ((double)s.nnzJ + (double)s.nnzLU);
        stats->levelFactorMs += lfMs;
        stats->levelFactorBytes += (double)levelSys * (double)sizeof(T) * ((double)s.nnzJ + (double)s.nnzLU);
        stats->tailMs += tMs;
    }
    cudaEventDestroy(evFork);
    for (auto& e : evJoin) cudaEventDestroy(e);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    if (ms) cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int NewtonDispatch(gs_grid* G, int count, bool useScale, bool startFromWs, const gs_pf_opts& o, float* ms,
                   NewtonStats* stats = nullptr, const double* vmSys = nullptr, const double* vaSys = nullptr) {
    G->view.qlimRevert = o.revert_q_limits ? 1 : 0;  // the call's Q-limit options (PowerFlowOptions.cs:101, 110)
    G->view.qlimMaxPasses = o.max_q_limit_passes > 0 ? o.max_q_limit_passes : kMaxQPasses;
    if (o.partial_pivoting) {  // every step by the per-system partial-pivoting factorisation (FP64)
        const bool was = G->gpMode;
        G->gpMode = true;
        const int rc = Newton<double>(G, count, useScale, startFromWs, o, ms, stats, vmSys, vaSys);
        G->gpMode = was;
        return rc;
    }
    if (o.precision == GS_PREC_MIXED) return Newton<float>(G, count, useScale, startFromWs, o, ms, stats, vmSys, vaSys);
    return Newton<double>(G, count, useScale, startFromWs, o, ms, stats, vmSys, vaSys);
}

// ---- the DC-angle retry (NewtonShell.SolveWithRetry, NewtonShell.cs:227-268) ----
constexpr double kRetryStallFactor = 1e-3;        // NewtonShell.cs:146
constexpr double kRetryLastStepFactor = 0.5;      // NewtonShell.cs:167
constexpr double kMaxRetryBranchAngleDeg = 90.0;  // NewtonShell.cs:142

int UploadGrid(gs_grid* G);

int RetryGridOf(gs_grid* G, gs_grid** out) {
    if (!G->rgrid) {
        auto R = std::make_unique<gs_grid>();
        R->ctx = G->ctx;
        R->host = G->host;
        std::string err = Analyze(R->host, R->sym, G->sym.qlim);
        if (!err.empty()) return SetErr(G->ctx, GS_ERR_INVALID_ARG, err);
        int rc = UploadGrid(R.get());
        if (rc) return rc;
        G->rgrid = std::move(R);
    }
    *out = G->rgrid.get();
    return GS_OK;
}

// The element-outage arrays of workspace w for systems 0 .. e.size()-1 (the rest: no change).
int UploadElements(gs_grid* G, Workspace& w, const std::vector<ElemSys>& e) {
    gs_ctx* ctx = G->ctx;
    const int B = w.B;
    std::vector<int> ob(2 * (size_t)B, -1), ot(2 * (size_t)B, 0), sb(B, -1);
    std::vector<double> ov(2 * (size_t)B, NAN), dp(B, 0.0), dq(B, 0.0), qn(B, 0.0), qx(B, 0.0);
    for (size_t k = 0; k < e.size(); k++) {
        for (int q = 0; q < 2; q++) { ob[2 * k + q] = e[k].ovBus[q]; ot[2 * k + q] = e[k].ovType[q]; ov[2 * k + q] = e[k].ovVm[q]; }
        sb[k] = e[k].specBus; dp[k] = e[k].dp; dq[k] = e[k].dq; qn[k] = e[k].qmin; qx[k] = e[k].qmax;
    }
    GS_CUDA(cudaMemcpy(w.ovBus.p, ob.data(), ob.size() * 4, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(w.ovType.p, ot.data(), ot.size() * 4, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(w.ovVm.p, ov.data(), ov.size() * 8, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(w.specBus.p, sb.data(), sb.size() * 4, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(w.specDp.p, dp.data(), dp.size() * 8, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(w.specDq.p, dq.data(), dq.size() * 8, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(w.specQmin.p, qn.data(), qn.size() * 8, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(w.specQmax.p, qx.data(), qx.size() * 8, cudaMemcpyHostToDevice));
    return GS_OK;
}

// The branches outage id `id` takes out: none (-1), one branch (id < nbr), or the set id - nbr of the installed table.
std::vector<int> OutageBranches(const gs_grid* G, int id) {
    if (id < 0) return {};
    if (id < G->sym.nbr) return {id};
    std::vector<int> b;
    const int* p = &G->sets.br[(size_t)(id - G->sym.nbr) * kSetBranches];
    for (int j = 0; j < kSetBranches; j++)
        if (p[j] >= 0) b.push_back(p[j]);
    return b;
}

// Install a call's outage sets on G: the kernels read them through G->view until UninstallSets.
int InstallSets(gs_grid* G, const OutageSetTable& t) {
    gs_ctx* ctx = G->ctx;
    G->sets = t;
    G->view.nSet = t.n;
    if (t.n == 0) return GS_OK;
    GS_CUDA(G->setBrBuf.alloc(t.br.size() * 4));
    GS_CUDA(G->setCellBuf.alloc(t.cell.size() * 4));
    GS_CUDA(G->setRedBuf.alloc(t.red.size() * 8));
    GS_CUDA(cudaMemcpy(G->setBrBuf.p, t.br.data(), t.br.size() * 4, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(G->setCellBuf.p, t.cell.data(), t.cell.size() * 4, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(G->setRedBuf.p, t.red.data(), t.red.size() * 8, cudaMemcpyHostToDevice));
    G->view.setBr = G->setBrBuf.as<int>();
    G->view.setCell = G->setCellBuf.as<int>();
    G->view.setRed = G->setRedBuf.as<double>();
    return GS_OK;
}

void UninstallSets(gs_grid* G) {
    G->sets = OutageSetTable();
    G->view.nSet = 0;
    if (G->rgrid) { G->rgrid->sets = OutageSetTable(); G->rgrid->view.nSet = 0; }
}

// The largest angle across an in-service branch (the outaged ones excluded), net of its phase shift, in
// [-180, 180] degrees (NewtonShell.MaxBranchAngleDeg).
double MaxBranchAngleDeg(const HostGrid& h, const std::vector<int>& skip, const double* vaRad, size_t stride) {
    double mx = 0.0;
    for (int k = 0; k < h.nbr; k++) {
        if (!h.brOn[k] || std::find(skip.begin(), skip.end(), k) != skip.end()) continue;
        const double a = (vaRad[h.brF[k] * stride] - vaRad[h.brT[k] * stride]) * 180.0 / 3.14159265358979323846 - h.shift[k];
        mx = std::max(mx, std::fabs(std::remainder(a, 360.0)));
    }
    return mx;
}

// After the Newton run of `count` systems in G's workspace (system s with outage[s], load scaling loadScale[s * n]
// when given, started warm from ws.startVm/startVa when `warm`): systems whose last Newton run failed to converge and
// stalled (NewtonShell.Stalled, :162 and :200-206) are solved again from DC power-flow angles (the magnitudes of the
// ordinary start), in a twin grid's workspace; a retry that converges with every branch angle within 90 degrees
// replaces the system's result (state, status, iterations, mismatch), any other keeps the first result.
int RetryStalled(gs_grid* G, int count, const int* outage, const double* loadScale, bool warm, const gs_pf_opts& o,
                 float* msOut, NewtonStats* stats) {
    if (!o.retry_from_dc_start || o.max_iterations <= 1 || count <= 0) return GS_OK;
    gs_ctx* ctx = G->ctx;
    const Symbolic& s = G->sym;
    const HostGrid& h = G->host;
    Workspace& w = G->ws;
    const bool qlim = s.qlim;
    std::vector<int> st(count), it(count), pass(qlim ? count : 0), qs(qlim ? count : 0);
    std::vector<double> fin(count), start(count), before(count);
    GS_CUDA(cudaMemcpy(st.data(), w.status.p, count * 4, cudaMemcpyDeviceToHost));
    GS_CUDA(cudaMemcpy(it.data(), w.iters.p, count * 4, cudaMemcpyDeviceToHost));
    GS_CUDA(cudaMemcpy(fin.data(), w.finalMis.p, count * 8, cudaMemcpyDeviceToHost));
    GS_CUDA(cudaMemcpy(start.data(), w.startMis.p, count * 8, cudaMemcpyDeviceToHost));
    GS_CUDA(cudaMemcpy(before.data(), w.beforeLast.p, count * 8, cudaMemcpyDeviceToHost));
    if (qlim) {
        GS_CUDA(cudaMemcpy(pass.data(), w.passIter.p, count * 4, cudaMemcpyDeviceToHost));
        GS_CUDA(cudaMemcpy(qs.data(), w.qState.p, count * 4, cudaMemcpyDeviceToHost));
    }
    int gridSlack = -1, slacks = 0;
    for (int i = 0; i < s.n; i++) if (s.type0[i] == 3) { gridSlack = i; slacks++; }
    if (slacks != 1) return GS_OK;  // TrySeedDcAngles needs exactly one slack
    const bool elems = !G->elemBatch.empty();
    auto slackOf = [&](int k) {  // an element outage may have moved the reference
        if (elems)
            for (int q = 0; q < 2; q++)
                if (G->elemBatch[k].ovBus[q] >= 0 && G->elemBatch[k].ovType[q] == 3) return G->elemBatch[k].ovBus[q];
        return gridSlack;
    };
    std::vector<int> cand;
    for (int k = 0; k < count; k++) {
        if (st[k] == GS_PF_CONVERGED) continue;
        if (qlim && (qs[k] & kQFinalConverged)) continue;  // the last run converged: the pass cap, not Newton, failed
        const int steps = qlim ? pass[k] : it[k];
        const bool diverged = st[k] == GS_PF_DIVERGED;
        const bool capReached = !diverged && st[k] != GS_PF_NON_FINITE && steps >= o.max_iterations;
        if (capReached && steps == 0) continue;
        if (fin[k] <= kRetryStallFactor * start[k]) continue;  // still converging (a NaN counts as stalled)
        if (capReached && steps >= 2 && fin[k] <= kRetryLastStepFactor * before[k]) continue;
        cand.push_back(k);
    }
    if (cand.empty()) return GS_OK;
    const int n = s.n;
    // ordinary start magnitudes, DC angles
    std::vector<double> vmBase(n), vaBase(n);
    if (warm) {
        GS_CUDA(cudaMemcpy(vmBase.data(), w.startVm.p, n * 8, cudaMemcpyDeviceToHost));
        GS_CUDA(cudaMemcpy(vaBase.data(), w.startVa.p, n * 8, cudaMemcpyDeviceToHost));
    } else {
        vmBase = s.vm0;
        vaBase = s.va0;
    }
    std::vector<int> ok, okOut;
    std::vector<std::vector<double>> seeds;
    for (int k : cand) {
        std::vector<double> th;
        const double* sc = loadScale ? loadScale + (size_t)k * n : nullptr;
        const int slack = slackOf(k);
        int dead = -1, specBus = -1;
        double dp = 0.0;
        if (elems) {
            const ElemSys& e = G->elemBatch[k];
            for (int q = 0; q < 2; q++) if (e.ovBus[q] >= 0 && e.ovType[q] == 0) dead = e.ovBus[q];
            specBus = e.specBus;
            dp = e.dp;
        }
        if (!DcAngles(h, s, OutageBranches(G, outage ? outage[k] : -1), slack, sc, th, dead, specBus, dp)) continue;
        std::vector<double> va(n);
        for (int i = 0; i < n; i++)
            va[i] = i == slack ? vaBase[slack] : vaBase[slack] + std::remainder(th[i], 360.0) * 3.14159265358979323846 / 180.0;
        seeds.push_back(std::move(va));
        ok.push_back(k);
        okOut.push_back(outage ? outage[k] : -1);
    }
    if (ok.empty()) return GS_OK;
    gs_grid* R = nullptr;
    int rc = RetryGridOf(G, &R);
    if (rc) return rc;
    if (G->view.nSet > 0 && (rc = InstallSets(R, G->sets)) != GS_OK) return rc;  // the same outage ids
    const int nc = (int)ok.size();
    const int B = std::max(32, (nc + 31) / 32 * 32);
    rc = EnsureWorkspace(R, B, o.precision, false, loadScale != nullptr);
    if (rc) return rc;
    Workspace& rw = R->ws;
    std::vector<int> outs(B, -1);
    for (int c = 0; c < nc; c++) outs[c] = okOut[c];
    GS_CUDA(cudaMemcpy(rw.outage.p, outs.data(), B * 4, cudaMemcpyHostToDevice));
    R->view.qlimOn = G->view.qlimOn;
    struct RetryOvOff { gs_grid* r; ~RetryOvOff() { r->ws.ovOn = r->tws.ovOn = r->mws.ovOn = false; r->elemBatch.clear(); } } retryOvOff{R};
    if (elems) {  // the retried systems keep their element outages
        R->elemBatch.clear();
        for (int c = 0; c < nc; c++) R->elemBatch.push_back(G->elemBatch[ok[c]]);
        if ((rc = UploadElements(R, rw, R->elemBatch)) != GS_OK) return rc;
        rw.ovOn = R->tws.ovOn = true;
    }
    if (loadScale) {
        std::vector<double> scl((size_t)n * B, 1.0);
        for (int c = 0; c < nc; c++)
            for (int i = 0; i < n; i++) scl[(size_t)i * B + c] = loadScale[(size_t)ok[c] * n + i];
        GS_CUDA(cudaMemcpy(rw.loadScale.p, scl.data(), scl.size() * 8, cudaMemcpyHostToDevice));
    }
    std::vector<double> vmS((size_t)n * B, 1.0), vaS((size_t)n * B, 0.0);
    for (int c = 0; c < nc; c++) {
        for (int i = 0; i < n; i++) {
            vmS[(size_t)i * B + c] = vmBase[i];
            vaS[(size_t)i * B + c] = seeds[c][i];
        }
        if (elems && !warm)  // a bus that starts PQ in this outage starts from its stored magnitude
            for (int q = 0; q < 2; q++) {
                const ElemSys& e = G->elemBatch[ok[c]];
                if (e.ovBus[q] >= 0 && e.ovType[q] == 1 && !std::isnan(e.ovVm[q])) vmS[(size_t)e.ovBus[q] * B + c] = e.ovVm[q];
            }
    }
    DevBuf dvm, dva;
    GS_CUDA(dvm.alloc(vmS.size() * 8));
    GS_CUDA(dva.alloc(vaS.size() * 8));
    GS_CUDA(cudaMemcpy(dvm.p, vmS.data(), vmS.size() * 8, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(dva.p, vaS.data(), vaS.size() * 8, cudaMemcpyHostToDevice));
    float ms = 0;
    rc = NewtonDispatch(R, nc, loadScale != nullptr, false, o, &ms, stats, dvm.as<double>(), dva.as<double>());
    if (rc) return rc;
    if (msOut) *msOut += ms;
    // keep the retries that converged within the branch-angle bound
    std::vector<int> rst(nc);
    std::vector<double> rva((size_t)n * B);
    GS_CUDA(cudaMemcpy(rst.data(), rw.status.p, nc * 4, cudaMemcpyDeviceToHost));
    GS_CUDA(cudaMemcpy(rva.data(), rw.va.p, rva.size() * 8, cudaMemcpyDeviceToHost));
    std::vector<int2> pairs;
    for (int c = 0; c < nc; c++)
        if (rst[c] == GS_PF_CONVERGED &&
            MaxBranchAngleDeg(h, OutageBranches(G, okOut[c]), rva.data() + c, (size_t)B) <= kMaxRetryBranchAngleDeg)
            pairs.push_back(make_int2(c, ok[c]));
    if (pairs.empty()) return GS_OK;
    DevBuf dp;
    GS_CUDA(dp.alloc(pairs.size() * sizeof(int2)));
    GS_CUDA(cudaMemcpy(dp.p, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice));
    const DevBatch from = MakeBatchWs(rw, R->sym.nLevels, rw.B, nc, loadScale != nullptr);
    const DevBatch to = MakeBatch(G, count, loadScale != nullptr);
    k_move_listed<<<dim3((n + 7) / 8, ((int)pairs.size() + 31) / 32), dim3(32, 8), 0, ctx->stream>>>(
        from, to, dp.as<int2>(), (int)pairs.size(), n);
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaStreamSynchronize(ctx->stream));
    return GS_OK;
}

// Systems of the batch whose static pivot collapsed (kFlagPivotPerturbed) are solved again from their start with row
// partial pivoting at every step (k_gp_solve, FP64, in the twin grid's workspace), as the reference factors every
// system (SparseLuFactorization.Factor, NewtonShell.SolveStep :74-120). A re-solve the factorisation carries to its
// end replaces the system's state, status, iterations and flags (kFlagPivoted); where the factorisation finds the
// matrix singular too, the system keeps its static result, still flagged. `outage` and `loadScale` are the batch's
// own arrays; `warm`: the batch started from ws.startVm / startVa.
int ResolvePivoted(gs_grid* G, int count, const int* outage, const double* loadScale, bool warm, const gs_pf_opts& o,
                   float* msOut) {
    if (count <= 0) return GS_OK;
    gs_ctx* ctx = G->ctx;
    const Symbolic& s = G->sym;
    Workspace& w = G->ws;
    std::vector<int> fl(count);
    GS_CUDA(cudaMemcpy(fl.data(), w.flags.p, count * 4, cudaMemcpyDeviceToHost));
    std::vector<int> cand;
    for (int k = 0; k < count; k++)
        if (fl[k] & kFlagPivotPerturbed) cand.push_back(k);
    if (cand.empty()) return GS_OK;
    gs_grid* R = nullptr;
    int rc = RetryGridOf(G, &R);
    if (rc) return rc;
    if (G->view.nSet > 0 && (rc = InstallSets(R, G->sets)) != GS_OK) return rc;  // the same outage ids
    R->view.qlimOn = G->view.qlimOn;
    struct Restore {
        gs_grid* r;
        ~Restore() { r->gpMode = false; r->ws.ovOn = r->tws.ovOn = r->mws.ovOn = false; r->elemBatch.clear(); }
    } restore{R};
    const bool elems = !G->elemBatch.empty();
    const int n = s.n;
    gs_pf_opts o64 = o;
    o64.precision = GS_PREC_FP64;
    constexpr int kChunk = 256;  // within the compact workspace of the few-systems path
    for (size_t c0 = 0; c0 < cand.size(); c0 += kChunk) {
        const int nc = (int)std::min<size_t>(kChunk, cand.size() - c0);
        const int B = std::max(32, (nc + 31) / 32 * 32);
        if ((rc = EnsureWorkspace(R, B, GS_PREC_FP64, false, loadScale != nullptr)) != GS_OK) return rc;
        Workspace& rw = R->ws;
        std::vector<int> outs(B, -1);
        for (int c = 0; c < nc; c++) outs[c] = outage ? outage[cand[c0 + c]] : -1;
        GS_CUDA(cudaMemcpy(rw.outage.p, outs.data(), B * 4, cudaMemcpyHostToDevice));
        if (elems) {
            R->elemBatch.clear();
            for (int c = 0; c < nc; c++) R->elemBatch.push_back(G->elemBatch[cand[c0 + c]]);
            if ((rc = UploadElements(R, rw, R->elemBatch)) != GS_OK) return rc;
            rw.ovOn = R->tws.ovOn = true;
        }
        if (loadScale) {
            std::vector<double> scl((size_t)n * B, 1.0);
            for (int c = 0; c < nc; c++)
                for (int i = 0; i < n; i++) scl[(size_t)i * B + c] = loadScale[(size_t)cand[c0 + c] * n + i];
            GS_CUDA(cudaMemcpy(rw.loadScale.p, scl.data(), scl.size() * 8, cudaMemcpyHostToDevice));
        }
        if (warm) {
            GS_CUDA(cudaMemcpy(rw.startVm.p, w.startVm.p, (size_t)n * 8, cudaMemcpyDeviceToDevice));
            GS_CUDA(cudaMemcpy(rw.startVa.p, w.startVa.p, (size_t)n * 8, cudaMemcpyDeviceToDevice));
        }
        R->gpMode = true;
        float ms = 0;
        rc = NewtonDispatch(R, nc, loadScale != nullptr, warm, o64, &ms);
        R->gpMode = false;
        if (rc) return rc;
        if (msOut) *msOut += ms;
        std::vector<int> rfl(nc);
        GS_CUDA(cudaMemcpy(rfl.data(), rw.flags.p, nc * 4, cudaMemcpyDeviceToHost));
        std::vector<int2> pairs;
        for (int c = 0; c < nc; c++)
            if (!(rfl[c] & kFlagPivotFailed)) pairs.push_back(make_int2(c, cand[c0 + c]));
        if (pairs.empty()) continue;
        DevBuf dp;
        GS_CUDA(dp.alloc(pairs.size() * sizeof(int2)));
        GS_CUDA(cudaMemcpy(dp.p, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice));
        const DevBatch from = MakeBatchWs(rw, R->sym.nLevels, rw.B, nc, loadScale != nullptr);
        const DevBatch to = MakeBatch(G, count, loadScale != nullptr);
        k_move_listed<<<dim3((n + 7) / 8, ((int)pairs.size() + 31) / 32), dim3(32, 8), 0, ctx->stream>>>(
            from, to, dp.as<int2>(), (int)pairs.size(), n);
        GS_CUDA(cudaGetLastError());
        GS_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return GS_OK;
}

int CheckOpts(gs_ctx* ctx, const gs_pf_opts* o) {
    if (!o) return SetErr(ctx, GS_ERR_INVALID_ARG, "null options");
    if (!(o->tolerance > 0) || o->tolerance > 1e-2) return SetErr(ctx, GS_ERR_INVALID_ARG, "tolerance must be in (0, 1e-2]");
    if (o->max_iterations < 0) return SetErr(ctx, GS_ERR_INVALID_ARG, "max_iterations must be 0 or more");
    if (!(o->diverge_limit_pu > 0)) return SetErr(ctx, GS_ERR_INVALID_ARG, "diverge_limit_pu must be above 0");
    if (o->precision != GS_PREC_FP64 && o->precision != GS_PREC_MIXED)
        return SetErr(ctx, GS_ERR_INVALID_ARG, "unknown precision");
    if (o->max_q_limit_passes < 0) return SetErr(ctx, GS_ERR_INVALID_ARG, "max_q_limit_passes must be 0 (the default) or more");
    if (o->post_fault_rating < GS_RATE_A || o->post_fault_rating > GS_RATE_C)
        return SetErr(ctx, GS_ERR_INVALID_ARG, "unknown post_fault_rating");
    return GS_OK;
}

int ChooseB(gs_grid* G, int want, const gs_pf_opts& o) {
    size_t freeB = 0, total = 0;
    cudaMemGetInfo(&freeB, &total);
    size_t per = PerSystemBytes(G->sym, o.precision);
    size_t cap = (size_t)(0.6 * (double)(freeB + (G->ws.lu.bytes + G->ws.vm.bytes + G->ws.va.bytes + G->ws.code.bytes +
                                                 G->ws.value.bytes + G->ws.y.bytes))) / per;
    int B = (int)std::min<size_t>(cap, (size_t)1 << 20);
    if (o.batch_width > 0) B = std::min(B, o.batch_width);
    if (o.partial_pivoting) B = std::min(B, 256);  // such batches step on the few-systems path's compact workspace
    B = std::min(B, ((want + 31) / 32) * 32);
    B = (B / 32) * 32;
    return std::max(B, 32);
}

// Solve the intact grid once in system 0 of the workspace (B = 32) and keep its state in startVm/Va.
// The grid analysed for Q-limit enforcement (the same host data; every PV bus has a Q equation in its pattern),
// built on the first call that enforces Q limits.
int QGridOf(gs_grid* G, gs_grid** out) {
    if (!G->qgrid) {
        auto Q = std::make_unique<gs_grid>();
        Q->ctx = G->ctx;
        Q->host = G->host;
        std::string err = Analyze(Q->host, Q->sym, true);
        if (!err.empty()) return SetErr(G->ctx, GS_ERR_INVALID_ARG, err);
        int rc = UploadGrid(Q.get());
        if (rc) return rc;
        G->qgrid = std::move(Q);
    }
    *out = G->qgrid.get();
    return GS_OK;
}

int SolveBase(gs_grid* G, const gs_pf_opts& o, int* status, int* iters, double* mis, float* ms) {
    gs_ctx* ctx = G->ctx;
    int rc = EnsureWorkspace(G, 32, o.precision, false, false);
    if (rc) return rc;
    std::vector<int> outage(G->ws.B, -1);
    GS_CUDA(cudaMemcpy(G->ws.outage.p, outage.data(), outage.size() * 4, cudaMemcpyHostToDevice));
    rc = NewtonDispatch(G, 1, false, false, o, ms);
    if (rc) return rc;
    const int none = -1;
    rc = ResolvePivoted(G, 1, &none, nullptr, false, o, ms);
    if (rc) return rc;
    rc = RetryStalled(G, 1, &none, nullptr, false, o, ms, nullptr);
    if (rc) return rc;
    const size_t B = G->ws.B;
    const int n = G->sym.n;
    // gather system 0 (strided) into the start arrays
    GS_CUDA(cudaMemcpy2D(G->ws.startVm.p, 8, G->ws.vm.p, B * 8, 8, n, cudaMemcpyDeviceToDevice));
    GS_CUDA(cudaMemcpy2D(G->ws.startVa.p, 8, G->ws.va.p, B * 8, 8, n, cudaMemcpyDeviceToDevice));
    GS_CUDA(cudaMemcpy(status, G->ws.status.p, 4, cudaMemcpyDeviceToHost));
    GS_CUDA(cudaMemcpy(iters, *status == GS_PF_CONVERGED ? G->ws.convIters.p : G->ws.iters.p, 4, cudaMemcpyDeviceToHost));
    GS_CUDA(cudaMemcpy(mis, G->ws.finalMis.p, 8, cudaMemcpyDeviceToHost));
    return GS_OK;
}

}  // namespace
}  // namespace gs

using namespace gs;

extern "C" {

namespace gs {
cudaError_t SetKernelAttributes();  // defined after the multi-grid kernels
bool ClusterWalkAvailable();
}

int gs_ctx_create(int device, const gs_ctx_opts* opts, gs_ctx** out) {
    if (!out) return GS_ERR_INVALID_ARG;
    *out = nullptr;
    int timeoutMs = (opts && opts->probe_timeout_ms > 0) ? opts->probe_timeout_ms : 10000;
    // The probe runs on a worker thread and is bounded (GpuContext.ProbeWithTimeout, GpuContext.cs:325-345).
    struct Probe { int rc = GS_ERR_TIMEOUT; std::string msg = "device probe timed out"; cudaStream_t stream = nullptr; };
    auto probe = std::make_shared<Probe>();
    auto done = std::make_shared<std::atomic<bool>>(false);
    std::thread th([probe, done, device]() {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
            probe->rc = GS_ERR_NO_DEVICE; probe->msg = "no CUDA device " + std::to_string(device);
        } else if (cudaSetDevice(device) != cudaSuccess) {
            probe->rc = GS_ERR_NO_DEVICE; probe->msg = "cudaSetDevice failed";
        } else {
            double* d = nullptr;
            double h = 0;
            cudaStream_t s = nullptr;
            if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess && cudaMalloc(&d, 8) == cudaSuccess) {
                gs::k_selftest<<<1, 1, 0, s>>>(d);
                if (cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, s) == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess &&
                    h == std::ldexp(1.0, -40)) {
                    probe->rc = GS_OK; probe->msg = ""; probe->stream = s;
                } else {
                    probe->rc = GS_ERR_NO_DEVICE; probe->msg = "FP64 self-test failed";
                }
                cudaFree(d);
            } else {
                probe->rc = GS_ERR_NO_DEVICE; probe->msg = "device allocation failed in the probe";
            }
        }
        done->store(true);
    });
    auto t0 = std::chrono::steady_clock::now();
    while (!done->load() && std::chrono::steady_clock::now() - t0 < std::chrono::milliseconds(timeoutMs))
        std::this_thread::sleep_for(std::chrono::milliseconds(2));
    if (!done->load()) { th.detach(); return GS_ERR_TIMEOUT; }
    th.join();
    if (probe->rc != GS_OK) return probe->rc;
    gs_ctx* c = new gs_ctx();
    c->device = device;
    c->stream = probe->stream;
    if (cudaSetDevice(device) != cudaSuccess || gs::SetKernelAttributes() != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->partStream[1], cudaStreamNonBlocking) != cudaSuccess) { delete c; return GS_ERR_CUDA; }
    if (cudaMallocHost(&c->pinnedCount, 4 * sizeof(int)) != cudaSuccess) { delete c; return GS_ERR_CUDA; }
    c->clusterOk = gs::ClusterWalkAvailable() && std::getenv("GS_NO_CLUSTER_TAIL") == nullptr;
    *out = c;
    return GS_OK;
}

int gs_ctx_destroy(gs_ctx* c) {
    if (!c) return GS_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    if (c->pinnedCount) cudaFreeHost(c->pinnedCount);
    if (c->stream) cudaStreamDestroy(c->stream);
    for (auto& ps : c->partStream) if (ps) cudaStreamDestroy(ps);
    delete c;
    return GS_OK;
}

int gs_last_error(gs_ctx* c, char* buf, size_t len) {
    if (!c || !buf || len == 0) return GS_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> l(c->mu);
    size_t k = std::min(len - 1, c->lastError.size());
    std::memcpy(buf, c->lastError.data(), k);
    buf[k] = 0;
    return GS_OK;
}

int gs_grid_create(gs_ctx* ctx, const gs_grid_desc* desc, gs_grid** out) {
    if (!ctx || !desc || !out) return GS_ERR_INVALID_ARG;
    *out = nullptr;
    auto G = std::make_unique<gs_grid>();
    G->ctx = ctx;
    std::string err = CopyGrid(desc, G->host);
    if (!err.empty()) return SetErr(ctx, GS_ERR_INVALID_ARG, err);
    err = Analyze(G->host, G->sym);
    if (!err.empty()) return SetErr(ctx, GS_ERR_INVALID_ARG, err);
    GS_CUDA(cudaSetDevice(ctx->device));
    int rc = UploadGrid(G.get());
    if (rc) return rc;
    *out = G.release();
    return GS_OK;
}

int gs_grid_destroy(gs_grid* g) {
    if (!g) return GS_ERR_INVALID_ARG;
    cudaSetDevice(g->ctx->device);
    delete g;
    return GS_OK;
}

int gs_grid_info_get(gs_grid* g, gs_grid_info* info) {
    if (!g || !info) return GS_ERR_INVALID_ARG;
    FillInfo(g->host, g->sym, info);
    return GS_OK;
}

int gs_grid_schedule_get(gs_grid* g, gs_schedule* out) {
    if (!g || !out) return GS_ERR_INVALID_ARG;
    *out = g->sched;
    return GS_OK;
}

int gs_grid_schedule_set(gs_grid* g, const gs_schedule* sc) {
    if (!g || !sc) return GS_ERR_INVALID_ARG;
    if (sc->factor_cut < 1 || sc->solve_cut < 1 || sc->tail_max < 1 || sc->subtree_cut < -1)
        return SetErr(g->ctx, GS_ERR_INVALID_ARG,
                      "schedule: factor_cut, solve_cut and tail_max must be at least 1, subtree_cut at least -1");
    gs_schedule c = *sc;
    c.tail_max = std::min(c.tail_max, kTailMaxSystems);
    SetSchedule(g, c);
    return GS_OK;
}

int gs_screen_tune(gs_grid* G0, int32_t nOut, const int32_t* idx, const gs_pf_opts* opts, gs_schedule* out) {
    if (!G0 || nOut <= 0 || !idx || !out) return GS_ERR_INVALID_ARG;
    gs_ctx* ctx = G0->ctx;
    int rc = CheckOpts(ctx, opts);
    if (rc) return rc;
    gs_pf_opts o = *opts;
    if (o.flat_start) return SetErr(ctx, GS_ERR_UNSUPPORTED, "flat_start: pass a flat start in the descriptor");
    if (o.partial_pivoting) return SetErr(ctx, GS_ERR_UNSUPPORTED, "partial_pivoting steps on no batched schedule");
    o.phase_timing = 0;
    GS_CUDA(cudaSetDevice(ctx->device));
    gs_grid* G = G0;
    if (o.enforce_q_limits && (rc = QGridOf(G0, &G)) != GS_OK) return rc;
    const Symbolic& s = G->sym;
    for (int k = 0; k < nOut; k++)
        if (idx[k] < 0 || idx[k] >= s.nbr || !G->host.brOn[idx[k]])
            return SetErr(ctx, GS_ERR_INVALID_ARG, "outage index out of range or out of service");
    G->view.qlimOn = o.enforce_q_limits ? 1 : 0;
    const bool warm = o.warm_start_from_base != 0;
    if (warm) {
        int bst = 0, bit = 0;
        double bmis = 0;
        float bms = 0;
        if ((rc = SolveBase(G, o, &bst, &bit, &bmis, &bms)) != GS_OK) return rc;
    }
    const int B = ChooseB(G, nOut, o);
    const int cnt = std::min(B, (int)nOut);
    if ((rc = EnsureWorkspace(G, B, o.precision, false, false)) != GS_OK) return rc;
    std::vector<int> outs(B, -1);
    std::copy(idx, idx + cnt, outs.begin());
    GS_CUDA(cudaMemcpy(G->ws.outage.p, outs.data(), (size_t)B * 4, cudaMemcpyHostToDevice));
    int timed = 0;
    // the sample's Newton batch under one schedule: the best device time of two runs
    auto run = [&](const gs_schedule& sc, float* best) -> int {
        SetSchedule(G, sc);
        *best = 3.0e38f;
        for (int r = 0; r < 2; r++) {
            float ms = 0;
            const int rc2 = NewtonDispatch(G, cnt, false, warm, o, &ms);
            if (rc2) return rc2;
            *best = std::min(*best, ms);
        }
        timed++;
        return GS_OK;
    };
    const gs_schedule before = G->sched;
    gs_schedule best = before;
    float base = 0;
    if ((rc = run(before, &base)) != GS_OK) return rc;
    float bestMs = base;
    // coordinate descent: the few-systems threshold, then the factorisation's cut, then the solves' cut, then the
    // subtree cut (off, or the levels whose subtrees hold at most 16, 64 or 256 KB of FP32 LU for a system group)
    const int tails[4] = {74, 148, kTailMaxSystems, kTailMaxSystems};
    const int cutOpts[4] = {1, 2, 4, 4};
    for (int dim = 0; dim < 4; dim++) {
        const gs_schedule start = best;
        int subOpts[4] = {-1, -1, -1, -1};
        if (dim == 3) {
            SetSchedule(G, start);  // the persistent walk's first level under the schedule so far
            subOpts[1] = SubtreeCutFor(G, 16.0 * 1024);
            subOpts[2] = SubtreeCutFor(G, 64.0 * 1024);
            subOpts[3] = SubtreeCutFor(G, 256.0 * 1024);
        }
        const int nOpt = dim == 3 ? 4 : 3;
        for (int k = 0; k < nOpt; k++) {
            gs_schedule c = start;
            if (dim == 0) c.tail_max = tails[k];
            else if (dim == 1) c.factor_cut = cutOpts[k];
            else if (dim == 2) c.solve_cut = cutOpts[k];
            else c.subtree_cut = subOpts[k];
            if (c.tail_max == start.tail_max && c.factor_cut == start.factor_cut && c.solve_cut == start.solve_cut &&
                c.subtree_cut == start.subtree_cut)
                continue;
            if (dim == 3 && k > 0 && subOpts[k] == subOpts[k - 1]) continue;
            float ms = 0;
            if ((rc = run(c, &ms)) != GS_OK) { SetSchedule(G, before); return rc; }
            if (ms < bestMs) { bestMs = ms; best = c; }
        }
    }
    best.candidates = timed;
    best.default_ms = base;
    best.tuned_ms = bestMs;
    SetSchedule(G, best);
    *out = best;
    return GS_OK;
}

int gs_pf_solve(gs_grid* G, const gs_pf_opts* opts, gs_pf_result* res) {
    if (!G || !res) return GS_ERR_INVALID_ARG;
    gs_ctx* ctx = G->ctx;
    int rc = CheckOpts(ctx, opts);
    if (rc) return rc;
    gs_pf_opts o = *opts;
    if (o.flat_start) return SetErr(ctx, GS_ERR_UNSUPPORTED, "flat_start: pass a flat start in the descriptor");
    GS_CUDA(cudaSetDevice(ctx->device));
    if (o.enforce_q_limits && (rc = QGridOf(G, &G)) != GS_OK) return rc;
    int st = 0, it = 0;
    double mis = 0;
    float ms = 0;
    rc = SolveBase(G, o, &st, &it, &mis, &ms);
    if (rc) return rc;
    res->status = st;
    res->iterations = it;
    res->max_mismatch = mis;
    const int n = G->sym.n, nb = G->sym.nbr;
    const size_t B = G->ws.B;
    std::vector<double> vm(n), va(n);
    GS_CUDA(cudaMemcpy(vm.data(), G->ws.startVm.p, n * 8, cudaMemcpyDeviceToHost));
    GS_CUDA(cudaMemcpy(va.data(), G->ws.startVa.p, n * 8, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++) {
        if (res->vm) res->vm[i] = vm[i];
        if (res->va_deg) res->va_deg[i] = va[i] * 180.0 / 3.14159265358979323846;
    }
    if (res->p_inj_mw || res->q_inj_mvar) {
        GS_CUDA(G->ws.pq.alloc(2 * (size_t)n * B * 8));
        DevBatch b = MakeBatch(G, 1, false);
        GS_CUDA(cudaMemset(b.active, 0, B * 4));
        int one = 1;
        GS_CUDA(cudaMemcpy(b.active, &one, 4, cudaMemcpyHostToDevice));
        double* P = G->ws.pq.as<double>();
        double* Q = P + (size_t)n * B;
        if (o.precision == GS_PREC_MIXED)
            k_mismatch_jac<float><<<dim3((n + 7) / 8, B / 32), dim3(32, 8), 0, ctx->stream>>>(G->view, b, 0, P, Q, nullptr, 0);
        else
            k_mismatch_jac<double><<<dim3((n + 7) / 8, B / 32), dim3(32, 8), 0, ctx->stream>>>(G->view, b, 0, P, Q, nullptr, 0);
        GS_CUDA(cudaStreamSynchronize(ctx->stream));
        std::vector<double> p(n), q(n);
        GS_CUDA(cudaMemcpy2D(p.data(), 8, P, B * 8, 8, n, cudaMemcpyDeviceToHost));
        GS_CUDA(cudaMemcpy2D(q.data(), 8, Q, B * 8, 8, n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; i++) {
            if (res->p_inj_mw) res->p_inj_mw[i] = p[i] * G->host.base;
            if (res->q_inj_mvar) res->q_inj_mvar[i] = q[i] * G->host.base;
        }
    }
    if (nb > 0 && (res->loading_pct || res->sf_mva || res->st_mva)) {
        DevBuf tmp;
        GS_CUDA(tmp.alloc((size_t)nb * 5 * 8));
        double* ld = tmp.as<double>();
        double* sf = ld + nb;
        double* sto = sf + 2 * (size_t)nb;
        DevBatch b = MakeBatch(G, 1, false);
        k_lineflows<<<(nb + 127) / 128, 128, 0, ctx->stream>>>(G->view, b, G->host.base, ld, sf, sto);
        GS_CUDA(cudaStreamSynchronize(ctx->stream));
        std::vector<double> h((size_t)nb * 5);
        GS_CUDA(cudaMemcpy(h.data(), ld, h.size() * 8, cudaMemcpyDeviceToHost));
        for (int k = 0; k < nb; k++) {
            if (res->loading_pct) res->loading_pct[k] = h[k];
            if (res->sf_mva) { res->sf_mva[2 * k] = h[nb + 2 * k]; res->sf_mva[2 * k + 1] = h[nb + 2 * k + 1]; }
            if (res->st_mva) { res->st_mva[2 * k] = h[3 * nb + 2 * k]; res->st_mva[2 * k + 1] = h[3 * nb + 2 * k + 1]; }
        }
    }
    return GS_OK;
}

int gs_pf_solve_batch(gs_grid* G, int32_t count, const double* loadScale, const int32_t* outage, const gs_pf_opts* opts,
                      int32_t* status, int32_t* iterations, double* maxMismatch, double* vmOut, double* vaOut) {
    if (!G || count < 0) return GS_ERR_INVALID_ARG;
    gs_ctx* ctx = G->ctx;
    int rc = CheckOpts(ctx, opts);
    if (rc) return rc;
    gs_pf_opts o = *opts;
    if (o.flat_start) return SetErr(ctx, GS_ERR_UNSUPPORTED, "flat_start: pass a flat start in the descriptor");
    if (o.enforce_q_limits) {
        GS_CUDA(cudaSetDevice(ctx->device));
        if ((rc = QGridOf(G, &G)) != GS_OK) return rc;
    }
    const Symbolic& s = G->sym;
    if (outage)
        for (int k = 0; k < count; k++)
            if (outage[k] >= s.nbr || (outage[k] >= 0 && !G->host.brOn[outage[k]]))
                return SetErr(ctx, GS_ERR_INVALID_ARG, "outage index out of range or out of service");
    GS_CUDA(cudaSetDevice(ctx->device));
    const int n = s.n;
    int done = 0;
    while (done < count) {
        int B = ChooseB(G, count - done, o);
        rc = EnsureWorkspace(G, B, o.precision, false, loadScale != nullptr);
        if (rc) return rc;
        int cnt = std::min(B, count - done);
        std::vector<int> out(B, -1);
        for (int k = 0; k < cnt; k++) out[k] = outage ? outage[done + k] : -1;
        GS_CUDA(cudaMemcpy(G->ws.outage.p, out.data(), B * 4, cudaMemcpyHostToDevice));
        if (loadScale) {
            std::vector<double> sc((size_t)n * B, 1.0);
            for (int k = 0; k < cnt; k++)
                for (int i = 0; i < n; i++) sc[(size_t)i * B + k] = loadScale[(size_t)(done + k) * n + i];
            GS_CUDA(cudaMemcpy(G->ws.loadScale.p, sc.data(), sc.size() * 8, cudaMemcpyHostToDevice));
        }
        float ms = 0;
        rc = NewtonDispatch(G, cnt, loadScale != nullptr, false, o, &ms);
        if (rc) return rc;
        rc = ResolvePivoted(G, cnt, out.data(), loadScale ? loadScale + (size_t)done * n : nullptr, false, o, &ms);
        if (rc) return rc;
        rc = RetryStalled(G, cnt, out.data(), loadScale ? loadScale + (size_t)done * n : nullptr, false, o, &ms, nullptr);
        if (rc) return rc;
        std::vector<int> st(cnt), it(cnt);
        std::vector<double> mis(cnt);
        GS_CUDA(cudaMemcpy(st.data(), G->ws.status.p, cnt * 4, cudaMemcpyDeviceToHost));
        GS_CUDA(cudaMemcpy(it.data(), G->ws.iters.p, cnt * 4, cudaMemcpyDeviceToHost));
        GS_CUDA(cudaMemcpy(mis.data(), G->ws.finalMis.p, cnt * 8, cudaMemcpyDeviceToHost));
        for (int k = 0; k < cnt; k++) {
            if (status) status[done + k] = st[k];
            if (iterations) iterations[done + k] = it[k];
            if (maxMismatch) maxMismatch[done + k] = mis[k];
        }
        if (vmOut || vaOut) {
            std::vector<double> v((size_t)n * B);
            for (int pass = 0; pass < 2; pass++) {
                double* dst = pass == 0 ? vmOut : vaOut;
                if (!dst) continue;
                GS_CUDA(cudaMemcpy(v.data(), pass == 0 ? G->ws.vm.p : G->ws.va.p, v.size() * 8, cudaMemcpyDeviceToHost));
                const double f = pass == 0 ? 1.0 : 180.0 / 3.14159265358979323846;
                for (int k = 0; k < cnt; k++)
                    for (int i = 0; i < n; i++) dst[(size_t)(done + k) * n + i] = v[(size_t)i * B + k] * f;
            }
        }
        done += cnt;
    }
    return GS_OK;
}

}  // extern "C"

namespace gs {
namespace {

// One outage of a screen: branches taken out together, and for an element outage (ScreenElementOutage,
// ContingencyAnalysis.cs:1355-1437) a generator or a bus (whose branches are listed too).
struct Element {
    std::vector<int> branches;
    int gen = -1;
    int bus = -1;
};

// The bus with the largest remaining unit by |Pg| (first in model order among ties) among the buses reachable from
// `seeds` over in-service branches not in `gone`, never through `removedBus`; -1 when none (ReelectReference
// :1440-1488).
int ReelectReference(const HostGrid& h, const std::vector<int>& seeds, const std::vector<uint8_t>& gone, int removedBus,
                     int removedGen) {
    std::vector<std::vector<int>> adj(h.n);
    for (int k = 0; k < h.nbr; k++)
        if (h.brOn[k] && !gone[k]) { adj[h.brF[k]].push_back(h.brT[k]); adj[h.brT[k]].push_back(h.brF[k]); }
    std::vector<uint8_t> reach(h.n, 0);
    std::vector<int> queue;
    for (int x : seeds) if (x != removedBus && !reach[x]) { reach[x] = 1; queue.push_back(x); }
    for (size_t q = 0; q < queue.size(); q++)
        for (int v : adj[queue[q]])
            if (v != removedBus && !reach[v]) { reach[v] = 1; queue.push_back(v); }
    int best = -1;
    for (int g = 0; g < h.ngen; g++) {
        if (!h.genOn[g] || g == removedGen || h.genBus[g] == removedBus || !reach[h.genBus[g]]) continue;
        if (best < 0 || std::fabs(h.pg[g]) > std::fabs(h.pg[best])) best = g;
    }
    return best < 0 ? -1 : h.genBus[best];
}

// The set point of bus i from its in-service units other than `removedGen` (the last one in model order sets it,
// NewtonShell.BuildBusSpec); NaN when none is left.
double SetPointOf(const HostGrid& h, int i, int removedGen) {
    double vg = NAN;
    for (int g = 0; g < h.ngen; g++)
        if (h.genOn[g] && g != removedGen && h.genBus[g] == i) vg = h.vg[g];
    return vg;
}

// The screen of a list of outages (empty: the intact grid, ScreenBaseCase; one branch: ScreenBranches; several:
// ScreenOutageCore over several indices, ContingencyAnalysis.cs:1087-1097; a generator or a bus: ScreenElementOutage).
int ScreenOutageLists(gs_grid* G, int nOut, const std::vector<Element>& els, const gs_pf_opts* opts,
                      gs_n1_result* res) {
    if (!G || !res || nOut < 0) return GS_ERR_INVALID_ARG;
    gs_ctx* ctx = G->ctx;
    int rc = CheckOpts(ctx, opts);
    if (rc) return rc;
    gs_pf_opts o = *opts;
    if (o.flat_start) return SetErr(ctx, GS_ERR_UNSUPPORTED, "flat_start: pass a flat start in the descriptor");
    bool anyElement = false;
    for (const Element& e : els) anyElement = anyElement || e.gen >= 0 || e.bus >= 0;
    // generator and bus outages change bus types: they run on the grid analysed with every bus's P and Q rows
    if (o.enforce_q_limits || anyElement) {
        GS_CUDA(cudaSetDevice(ctx->device));
        if ((rc = QGridOf(G, &G)) != GS_OK) return rc;
    }
    G->view.qlimOn = o.enforce_q_limits ? 1 : 0;
    struct QlimRestore { gs_grid* g; ~QlimRestore() { g->view.qlimOn = g->view.qlim; } } qlimRestore{G};
    const Symbolic& s = G->sym;
    const HostGrid& h = G->host;
    // outage ids: -1, a branch, or nbr + the position of a multi-branch set in this call's table
    std::vector<int> ids(nOut, -1);
    OutageSetTable table;
    std::vector<std::vector<int>> lists(nOut);
    for (int k = 0; k < nOut; k++) lists[k] = els[k].branches;
    for (int k = 0; k < nOut; k++) {
        const std::vector<int>& b = lists[k];
        if ((int)b.size() > kSetBranches)
            return SetErr(ctx, GS_ERR_UNSUPPORTED, "an outage takes at most " + std::to_string(kSetBranches) + " branches");
        for (size_t j = 0; j < b.size(); j++) {
            // AN-02: an out-of-service branch is refused (ContingencyAnalysis.cs:290-300)
            if (b[j] < 0 || b[j] >= s.nbr || !h.brOn[b[j]])
                return SetErr(ctx, GS_ERR_INVALID_ARG, "branch " + std::to_string(b[j]) + " is not an in-service branch");
            for (size_t q = 0; q < j; q++)
                if (b[q] == b[j])
                    return SetErr(ctx, GS_ERR_INVALID_ARG, "branch " + std::to_string(b[j]) + " appears twice in one outage");
        }
        ids[k] = b.empty() ? -1 : b.size() == 1 ? b[0] : s.nbr + AddOutageSet(s, b, table);
    }
    const int* idx = ids.data();
    // element outages: bus type changes, lost output, a reference moved when its last unit goes (ReelectReference)
    std::vector<ElemSys> elem(anyElement ? nOut : 0);
    std::vector<ElementCut> cuts(anyElement ? nOut : 0);
    std::vector<uint8_t> noReference(nOut, 0);
    for (int k = 0; k < nOut && anyElement; k++) {
        const Element& e = els[k];
        ElemSys& x = elem[k];
        ElementCut& c = cuts[k];
        c.branches = e.branches;
        c.gen = e.gen;
        c.bus = e.bus;
        const bool warmStart = o.warm_start_from_base != 0;
        if (e.gen >= 0) {
            if (e.gen >= h.ngen || !h.genOn[e.gen])
                return SetErr(ctx, GS_ERR_INVALID_ARG, "generator " + std::to_string(e.gen) + " is not an in-service unit");
            const int i = h.genBus[e.gen];
            x.specBus = i;
            x.dp = h.pg[e.gen] / h.base;
            x.dq = h.qg[e.gen] / h.base;
            int left = 0;
            for (int g = 0; g < h.ngen; g++)
                if (h.genOn[g] && g != e.gen && h.genBus[g] == i) { left++; x.qmin += h.qmin[g]; x.qmax += h.qmax[g]; }
            const double vg = SetPointOf(h, i, e.gen);
            if (s.type0[i] == 3 && left == 0) {  // the reference's last unit: the reference moves
                const int j = ReelectReference(h, {i}, std::vector<uint8_t>(h.nbr, 0), -1, e.gen);
                if (j < 0) { noReference[k] = 1; continue; }
                x.ovBus[0] = i; x.ovType[0] = 1; x.ovVm[0] = warmStart ? NAN : h.vm[i];
                x.ovBus[1] = j; x.ovType[1] = 3; x.ovVm[1] = SetPointOf(h, j, e.gen);
                c.slackFrom = i;
                c.slackTo = j;
            } else if (s.type0[i] == 2 && left == 0) {  // a PV bus left with no unit is solved as PQ
                x.ovBus[0] = i; x.ovType[0] = 1; x.ovVm[0] = warmStart ? NAN : h.vm[i];
            } else if ((s.type0[i] == 2 || s.type0[i] == 3) && vg != s.vm0[i]) {  // the set point of the units left
                x.ovBus[0] = i; x.ovType[0] = s.type0[i]; x.ovVm[0] = vg;
            }
        } else if (e.bus >= 0) {
            x.ovBus[0] = e.bus; x.ovType[0] = 0;
            if (s.type0[e.bus] == 3) {  // the reference bus itself: the reference moves, seen from its neighbours
                std::vector<uint8_t> gone(h.nbr, 0);
                std::vector<int> seeds;
                for (int b : e.branches) {
                    gone[b] = 1;
                    seeds.push_back(h.brF[b] == e.bus ? h.brT[b] : h.brF[b]);
                }
                const int j = ReelectReference(h, seeds, gone, e.bus, -1);
                if (j < 0) { noReference[k] = 1; continue; }
                x.ovBus[1] = j; x.ovType[1] = 3; x.ovVm[1] = SetPointOf(h, j, -1);
                c.slackFrom = e.bus;
                c.slackTo = j;
            }
        }
    }
    GS_CUDA(cudaSetDevice(ctx->device));
    if ((rc = InstallSets(G, table)) != GS_OK) return rc;
    struct Uninstall { gs_grid* g; ~Uninstall() { UninstallSets(g); } } uninstall{G};
    struct OvOff { gs_grid* g; ~OvOff() { g->ws.ovOn = g->tws.ovOn = g->mws.ovOn = false; g->elemBatch.clear(); } } ovOff{G};
    const int n = s.n, nItems = s.nbr + h.nBnd + s.n;
    // the topology pass (ScreenStateCore :1118-1127): provably unsolvable states are reported without a solve,
    // and a state that does not converge says whether the outage split the network (:1661-1665)
    std::vector<uint8_t> splits(nOut), unsolv(nOut);
    {
        std::vector<int> single(nOut);
        for (int k = 0; k < nOut; k++) single[k] = idx[k] < s.nbr ? idx[k] : -1;
        std::string terr = OutageTopology(h, o.tolerance, nOut, single.data(), splits.data(), unsolv.data());
        for (int k = 0; k < nOut && terr.empty(); k++) {
            const bool isElement = anyElement && (els[k].gen >= 0 || els[k].bus >= 0);
            if (idx[k] < s.nbr && !isElement) continue;
            bool sp = false, un = false;
            ElementCut cut;
            if (isElement) cut = cuts[k];
            else cut.branches = lists[k];
            terr = ElementTopology(h, o.tolerance, cut, sp, un);
            splits[k] = sp;
            unsolv[k] = un || noReference[k];  // no unit left to take the reference: not solved (:1370-1372)
        }
        if (!terr.empty()) return SetErr(ctx, GS_ERR_INVALID_ARG, terr);
    }
    std::vector<int> solvePos;
    solvePos.reserve(nOut);
    for (int j = 0; j < nOut; j++) {
        if (!unsolv[j]) { solvePos.push_back(j); continue; }
        if (res->status) res->status[j] = GS_PF_UNSOLVABLE_PART;
        if (res->iterations) res->iterations[j] = 0;
        if (res->max_mismatch) res->max_mismatch[j] = 0.0;
        if (res->max_loading_pct) res->max_loading_pct[j] = 0.0;
        if (res->worst_boundary_pct) res->worst_boundary_pct[j] = 0.0;
        if (res->min_vm) res->min_vm[j] = 0.0;
        if (res->max_vm) res->max_vm[j] = 0.0;
        if (res->islanded) res->islanded[j] = splits[j];
        if (res->vm) std::fill(res->vm + (size_t)j * n, res->vm + (size_t)(j + 1) * n, 0.0);
        if (res->va_deg) std::fill(res->va_deg + (size_t)j * n, res->va_deg + (size_t)(j + 1) * n, 0.0);
    }
    const int nSolve = (int)solvePos.size();
    res->base_status = GS_PF_NOT_RUN;
    res->base_iterations = 0;
    res->n_singular_pivot = 0;
    res->n_partial_pivot = 0;
    res->n_batches = 0;
    double totalMs = 0;
    bool warm = false;
    if (o.warm_start_from_base) {
        int st = 0, it = 0;
        double mis = 0;
        float ms = 0;
        rc = SolveBase(G, o, &st, &it, &mis, &ms);
        if (rc) return rc;
        totalMs += ms;
        res->base_status = st;
        res->base_iterations = it;
        warm = st == GS_PF_CONVERGED;
    }
    // effective voltage limits (VoltageLimits.OperationalLowFor / HighFor, :55-67)
    bool perBus = false;
    if (o.per_bus_voltage_limits)
        for (int i = 0; i < n; i++) if (!std::isnan(h.vmin[i]) || !std::isnan(h.vmax[i])) perBus = true;
    std::vector<double> lo(n, 0.94), hi(n, 1.06);
    if (perBus)
        for (int i = 0; i < n; i++) {
            if (!std::isnan(h.vmin[i])) lo[i] = h.vmin[i];
            if (!std::isnan(h.vmax[i])) hi[i] = h.vmax[i];
        }
    DevBuf dlo, dhi, dbusId;
    GS_CUDA(dlo.alloc(n * 8)); GS_CUDA(dhi.alloc(n * 8)); GS_CUDA(dbusId.alloc(n * 4));
    GS_CUDA(cudaMemcpy(dlo.p, lo.data(), n * 8, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(dhi.p, hi.data(), n * 8, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(dbusId.p, h.busId.data(), n * 4, cudaMemcpyHostToDevice));
    const int chunk = 256;
    const int nChunks = (nItems + chunk - 1) / chunk;
    NewtonStats stats;
    int written = 0;
    bool capacityOk = true;
    int done = 0;
    while (done < nSolve) {
        int B = ChooseB(G, nSolve - done, o);
        rc = EnsureWorkspace(G, B, o.precision, true, false);
        if (rc) return rc;
        Workspace& w = G->ws;
        const size_t Bz = (size_t)B;
        const int cnt = std::min(B, nSolve - done);
        std::vector<int> out(B, -1);
        for (int k = 0; k < cnt; k++) out[k] = idx[solvePos[done + k]];
        GS_CUDA(cudaMemcpy(w.outage.p, out.data(), B * 4, cudaMemcpyHostToDevice));
        if (anyElement) {
            G->elemBatch.assign(cnt, ElemSys());
            for (int k = 0; k < cnt; k++) G->elemBatch[k] = elem[solvePos[done + k]];
            if ((rc = UploadElements(G, G->ws, G->elemBatch)) != GS_OK) return rc;
            G->ws.ovOn = G->tws.ovOn = true;
        }
        float ms = 0;
        rc = NewtonDispatch(G, cnt, false, warm, o, &ms, &stats);
        if (rc) return rc;
        rc = ResolvePivoted(G, cnt, out.data(), nullptr, warm, o, &ms);
        if (rc) return rc;
        rc = RetryStalled(G, cnt, out.data(), nullptr, warm, o, &ms, &stats);
        if (rc) return rc;
        totalMs += ms;
        res->n_batches++;
        stats.launches += 2;  // classification and compaction
        // classification of converged systems (its device time counts in the screen's device_ms)
        GS_CUDA(w.chunkCount.alloc((size_t)nChunks * Bz * 4));
        GS_CUDA(w.chunkOffset.alloc((size_t)nChunks * Bz * 4));
        EventPair clsEv, cmpEv;
        GS_CUDA(clsEv.create());
        GS_CUDA(cmpEv.create());
        GS_CUDA(cudaEventRecord(clsEv.a, ctx->stream));
        GS_CUDA(cudaMemsetAsync(w.chunkCount.p, 0, (size_t)nChunks * Bz * 4, ctx->stream));
        GS_CUDA(cudaMemsetAsync(w.maxLoad.p, 0, Bz * 8, ctx->stream));
        GS_CUDA(cudaMemsetAsync(w.minVmNeg.p, 0, Bz * 8, ctx->stream));
        GS_CUDA(cudaMemsetAsync(w.maxVmB.p, 0, Bz * 8, ctx->stream));
        GS_CUDA(cudaMemsetAsync(w.worstBnd.p, 0, Bz * 8, ctx->stream));
        Classify c{dlo.as<double>(), dhi.as<double>(), w.code.as<uint8_t>(), w.value.as<double>(),
                   w.maxLoad.as<unsigned long long>(), w.minVmNeg.as<unsigned long long>(),
                   w.maxVmB.as<unsigned long long>(), w.worstBnd.as<unsigned long long>(), w.chunkCount.as<int>(),
                   chunk, o.post_fault_rating};
        DevBatch b = MakeBatch(G, cnt, false);
        k_classify<<<dim3((nItems + 7) / 8, B / 32), dim3(32, 8), 0, ctx->stream>>>(G->view, b, c);
        GS_CUDA(cudaGetLastError());
        GS_CUDA(cudaEventRecord(clsEv.b, ctx->stream));
        std::vector<int> cc((size_t)nChunks * Bz), off((size_t)nChunks * Bz);
        GS_CUDA(cudaMemcpyAsync(cc.data(), w.chunkCount.p, cc.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
        std::vector<int> st(cnt), it(cnt), fl(cnt);
        std::vector<double> mis(cnt);
        std::vector<unsigned long long> mxl(cnt), mnv(cnt), mxv(cnt), wbd(cnt);
        GS_CUDA(cudaMemcpyAsync(st.data(), w.status.p, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CUDA(cudaMemcpyAsync(it.data(), w.iters.p, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
        std::vector<int> itc(cnt);
        GS_CUDA(cudaMemcpyAsync(itc.data(), w.convIters.p, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CUDA(cudaMemcpyAsync(fl.data(), w.flags.p, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CUDA(cudaMemcpyAsync(mis.data(), w.finalMis.p, cnt * 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CUDA(cudaMemcpyAsync(mxl.data(), w.maxLoad.p, cnt * 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CUDA(cudaMemcpyAsync(mnv.data(), w.minVmNeg.p, cnt * 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CUDA(cudaMemcpyAsync(mxv.data(), w.maxVmB.p, cnt * 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CUDA(cudaMemcpyAsync(wbd.data(), w.worstBnd.p, cnt * 8, cudaMemcpyDeviceToHost, ctx->stream));
        GS_CUDA(cudaStreamSynchronize(ctx->stream));
        totalMs += clsEv.ms();
        int batchTotal = 0;
        std::vector<int> sysStart(cnt);
        for (int k = 0; k < cnt; k++) {
            sysStart[k] = batchTotal;
            int acc = batchTotal;
            for (int ch = 0; ch < nChunks; ch++) {
                off[(size_t)ch * Bz + k] = acc;
                acc += cc[(size_t)ch * Bz + k];
            }
            batchTotal = acc;
        }
        for (int k = 0; k < cnt; k++) {
            const int g = solvePos[done + k];
            auto asD = [](unsigned long long u) { double d; std::memcpy(&d, &u, 8); return d; };
            const bool conv = st[k] == GS_PF_CONVERGED;
            if (res->status) res->status[g] = st[k];
            if (res->iterations) res->iterations[g] = conv ? itc[k] : it[k];
            if (res->max_mismatch) res->max_mismatch[g] = mis[k];
            if (res->max_loading_pct) res->max_loading_pct[g] = conv ? asD(mxl[k]) : 0.0;
            if (res->min_vm) res->min_vm[g] = conv ? 100.0 - asD(mnv[k]) : 0.0;
            if (res->max_vm) res->max_vm[g] = conv ? asD(mxv[k]) : 0.0;
            if (res->worst_boundary_pct) res->worst_boundary_pct[g] = conv ? asD(wbd[k]) : 0.0;
            if (res->islanded) res->islanded[g] = !conv && splits[g];
            if (res->viol_ptr) res->viol_ptr[g] = written + sysStart[k];
            if (fl[k] & kFlagPivotPerturbed) res->n_singular_pivot++;
            if (fl[k] & kFlagPivoted) res->n_partial_pivot++;
        }
        if (written + batchTotal > res->viol_capacity || !res->viol_kind || !res->viol_element || !res->viol_value) {
            capacityOk = false;
        } else if (batchTotal > 0) {
            GS_CUDA(cudaMemcpy(w.chunkOffset.p, off.data(), off.size() * 4, cudaMemcpyHostToDevice));
            GS_CUDA(w.outKind.alloc((size_t)batchTotal * 4));
            GS_CUDA(w.outElem.alloc((size_t)batchTotal * 4));
            GS_CUDA(w.outVal.alloc((size_t)batchTotal * 8));
            GS_CUDA(cudaEventRecord(cmpEv.a, ctx->stream));
            k_compact<<<dim3((nChunks + 3) / 4, B / 32), dim3(32, 4), 0, ctx->stream>>>(
                G->view, b, c, w.chunkOffset.as<int>(), w.outKind.as<int>(), w.outElem.as<int>(), w.outVal.as<double>(),
                dbusId.as<int>());
            GS_CUDA(cudaGetLastError());
            GS_CUDA(cudaEventRecord(cmpEv.b, ctx->stream));
            GS_CUDA(cudaMemcpyAsync(res->viol_kind + written, w.outKind.p, (size_t)batchTotal * 4, cudaMemcpyDeviceToHost, ctx->stream));
            GS_CUDA(cudaMemcpyAsync(res->viol_element + written, w.outElem.p, (size_t)batchTotal * 4, cudaMemcpyDeviceToHost, ctx->stream));
            GS_CUDA(cudaMemcpyAsync(res->viol_value + written, w.outVal.p, (size_t)batchTotal * 8, cudaMemcpyDeviceToHost, ctx->stream));
            GS_CUDA(cudaStreamSynchronize(ctx->stream));
            totalMs += cmpEv.ms();
        }
        written += batchTotal;
        if (res->vm || res->va_deg) {
            std::vector<double> v((size_t)n * Bz);
            for (int pass = 0; pass < 2; pass++) {
                double* dst = pass == 0 ? res->vm : res->va_deg;
                if (!dst) continue;
                GS_CUDA(cudaMemcpy(v.data(), pass == 0 ? w.vm.p : w.va.p, v.size() * 8, cudaMemcpyDeviceToHost));
                const double f = pass == 0 ? 1.0 : 180.0 / 3.14159265358979323846;
                for (int k = 0; k < cnt; k++)
                    for (int i = 0; i < n; i++) dst[(size_t)solvePos[done + k] * n + i] = v[(size_t)i * Bz + k] * f;
            }
        }
        done += cnt;
    }
    if (res->viol_ptr) {  // a state reported without a solve has no entries: it starts where the next one does
        res->viol_ptr[nOut] = written;
        for (int j = nOut - 1; j >= 0; j--)
            if (unsolv[j]) res->viol_ptr[j] = res->viol_ptr[j + 1];
    }
    res->viol_count = written;
    res->device_ms = totalMs;
    res->kernel_launches = stats.launches;
    res->newton_iterations = stats.iterations;
    res->factor_ms = stats.factorMs;
    res->solve_ms = stats.solveMs;
    res->mismatch_ms = stats.mismatchMs;
    res->other_ms = stats.otherMs;
    res->factor_bytes = stats.factorBytes;
    res->level_factor_ms = stats.levelFactorMs;
    res->level_factor_bytes = stats.levelFactorBytes;
    res->tail_ms = stats.tailMs;
    return capacityOk ? GS_OK : GS_ERR_CAPACITY;
}

}  // namespace
}  // namespace gs

extern "C" {

int gs_n1_screen(gs_grid* G, int32_t nOut, const int32_t* idx, const gs_pf_opts* opts, gs_n1_result* res) {
    if (!G || !res || nOut < 0 || (nOut > 0 && !idx)) return GS_ERR_INVALID_ARG;
    std::vector<Element> lists(nOut);
    for (int k = 0; k < nOut; k++) {
        if (idx[k] < -1)
            return SetErr(G->ctx, GS_ERR_INVALID_ARG, "branch " + std::to_string(idx[k]) + " is not an in-service branch");
        if (idx[k] >= 0) lists[k].branches.push_back(idx[k]);
    }
    return ScreenOutageLists(G, nOut, lists, opts, res);
}

int gs_nk_screen(gs_grid* G, int32_t nOut, int32_t k, const int32_t* sets, const gs_pf_opts* opts, gs_n1_result* res) {
    if (!G || !res || nOut < 0 || k < 1 || (nOut > 0 && !sets)) return GS_ERR_INVALID_ARG;
    std::vector<Element> lists(nOut);
    for (int j = 0; j < nOut; j++)
        for (int q = 0; q < k; q++) {
            const int b = sets[(size_t)j * k + q];
            if (b < -1)
                return SetErr(G->ctx, GS_ERR_INVALID_ARG, "branch " + std::to_string(b) + " is not an in-service branch");
            if (b >= 0) lists[j].branches.push_back(b);
        }
    return ScreenOutageLists(G, nOut, lists, opts, res);
}

int gs_element_screen(gs_grid* G, int32_t nOut, const int32_t* kind, const int32_t* index, const gs_pf_opts* opts,
                      gs_n1_result* res) {
    if (!G || !res || nOut < 0 || (nOut > 0 && (!kind || !index))) return GS_ERR_INVALID_ARG;
    const HostGrid& h = G->host;
    std::vector<Element> els(nOut);
    for (int j = 0; j < nOut; j++) {
        const int x = index[j];
        switch (kind[j]) {
            case GS_OUTAGE_BRANCH:
                if (x < 0 || x >= h.nbr || !h.brOn[x])
                    return SetErr(G->ctx, GS_ERR_INVALID_ARG, "branch " + std::to_string(x) + " is not an in-service branch");
                els[j].branches.push_back(x);
                break;
            case GS_OUTAGE_GENERATOR:
                if (x < 0 || x >= h.ngen || !h.genOn[x])
                    return SetErr(G->ctx, GS_ERR_INVALID_ARG, "generator " + std::to_string(x) + " is not an in-service unit");
                els[j].gen = x;
                break;
            case GS_OUTAGE_BUS:
                if (x < 0 || x >= h.n) return SetErr(G->ctx, GS_ERR_INVALID_ARG, "bus position " + std::to_string(x) + " is out of range");
                els[j].bus = x;
                for (int k = 0; k < h.nbr; k++)  // the bus goes with every branch touching it (:1393-1399)
                    if (h.brOn[k] && (h.brF[k] == x || h.brT[k] == x)) els[j].branches.push_back(k);
                break;
            default:
                return SetErr(G->ctx, GS_ERR_INVALID_ARG, "unknown outage kind " + std::to_string(kind[j]));
        }
    }
    return ScreenOutageLists(G, nOut, els, opts, res);
}

}  // extern "C"

namespace gs {
namespace {

constexpr int kMaxPatterns = 8;  // analysed patterns kept per context

uint64_t PatternHash(int n, const int* rp, const int* ci) {  // FNV-1a over the pattern's integers
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](int v) {
        for (int q = 0; q < 4; q++) { h ^= (uint8_t)((uint32_t)v >> (8 * q)); h *= 1099511628211ull; }
    };
    mix(n);
    for (int i = 0; i <= n; i++) mix(rp[i]);
    for (int p = 0; p < rp[n]; p++) mix(ci[p]);
    return h;
}

// The analysed pattern of a (validated) CSR matrix: from the context's cache, or analysed and uploaded now.
// A row order whose diagonal is structurally zero-free: rowAt[c] = the row placed at position c. Empty when every row
// holds its own diagonal entry (the order is the identity); else a maximum transversal grown from the rows that do,
// by augmenting paths (depth first, iterative); {-1} when the pattern has none (structurally singular: the static
// pivots then report every system of it singular). The reference pivots by rows instead (SparseLuFactorization.cs:
// 69-195); with a zero-free diagonal the static diagonal pivots of the analysed order take the place of that choice.
std::vector<int> RowTransversal(int n, const int* rp, const int* ci) {
    std::vector<int> rowOfCol(n, -1), colOfRow(n, -1);
    bool full = true;
    for (int i = 0; i < n; i++) {
        for (int p = rp[i]; p < rp[i + 1]; p++)
            if (ci[p] == i) { rowOfCol[i] = i; colOfRow[i] = i; }
        full = full && colOfRow[i] == i;
    }
    if (full) return {};
    std::vector<int> mark(n, -1), via(n, -1), next(n, 0), path;
    for (int r0 = 0; r0 < n; r0++) {
        if (colOfRow[r0] >= 0) continue;
        path.assign(1, r0);
        next[r0] = rp[r0];
        int found = -1;
        while (!path.empty() && found < 0) {  // path: r0 and the rows reached from it through matched columns
            const int u = path.back();
            if (next[u] == rp[u + 1]) { path.pop_back(); continue; }
            const int c = ci[next[u]++];
            if (mark[c] == r0) continue;
            mark[c] = r0;
            if (rowOfCol[c] < 0) { found = c; break; }
            const int w = rowOfCol[c];
            via[w] = c;
            next[w] = rp[w];
            path.push_back(w);
        }
        if (found < 0) return {-1};
        for (int k = (int)path.size() - 1, c = found; k >= 0; k--) {  // each row on the path takes the next column
            const int u = path[k];
            colOfRow[u] = c;
            rowOfCol[c] = u;
            c = k > 0 ? via[u] : -1;
        }
    }
    return rowOfCol;
}

int PatternOf(gs_ctx* ctx, int n, const int* rp, const int* ci, MatrixPattern** out) {
    const uint64_t h = PatternHash(n, rp, ci);
    auto& v = ctx->patterns;
    for (size_t i = 0; i < v.size(); i++) {
        const MatrixPattern& P = *v[i];
        if (P.hash == h && P.n == n && std::equal(P.rowPtr.begin(), P.rowPtr.end(), rp) &&
            std::equal(P.colIdx.begin(), P.colIdx.end(), ci)) {
            std::rotate(v.begin() + i, v.begin() + i + 1, v.end());
            *out = v.back().get();
            return GS_OK;
        }
    }
    auto P = std::make_unique<MatrixPattern>();
    P->hash = h;
    P->n = n;
    P->rowPtr.assign(rp, rp + n + 1);
    P->colIdx.assign(ci, ci + rp[n]);
    P->grid = std::make_unique<gs_grid>();
    P->grid->ctx = ctx;
    // rows reordered to a zero-free diagonal where needed: the analysis runs on that order; a stored entry keeps its
    // slot through the map below and b's row i goes where row i went (the unknowns keep their order)
    const std::vector<int> rowAt = RowTransversal(n, rp, ci);
    const bool permuted = !rowAt.empty() && rowAt[0] >= 0;
    std::vector<int> rp2, ci2, posOfRow;
    if (permuted) {
        rp2.assign(n + 1, 0);
        posOfRow.assign(n, 0);
        for (int c = 0; c < n; c++) {
            const int r = rowAt[c];
            posOfRow[r] = c;
            rp2[c + 1] = rp2[c] + (rp[r + 1] - rp[r]);
            ci2.insert(ci2.end(), ci + rp[r], ci + rp[r + 1]);
        }
    }
    std::vector<int> slot2;
    const std::string err = permuted ? AnalyzeMatrix(n, rp2.data(), ci2.data(), P->grid->sym, slot2)
                                     : AnalyzeMatrix(n, rp, ci, P->grid->sym, P->aSlot);
    if (!err.empty()) return SetErr(ctx, GS_ERR_INVALID_ARG, err);
    int rc = UploadGrid(P->grid.get());
    if (rc) return rc;
    std::vector<int> pinv = P->grid->sym.pinv;  // right-hand-side row -> pivot position
    if (permuted) {
        P->aSlot.assign(rp[n], 0);
        for (int i = 0; i < n; i++)
            for (int p = rp[i]; p < rp[i + 1]; p++) P->aSlot[p] = slot2[rp2[posOfRow[i]] + (p - rp[i])];
        for (int i = 0; i < n; i++) pinv[i] = P->grid->sym.pinv[posOfRow[i]];
    }
    GS_CUDA(P->dSlot.alloc(std::max<size_t>(4, P->aSlot.size() * 4)));
    GS_CUDA(P->dPinv.alloc(pinv.size() * 4));
    if (!P->aSlot.empty()) GS_CUDA(cudaMemcpy(P->dSlot.p, P->aSlot.data(), P->aSlot.size() * 4, cudaMemcpyHostToDevice));
    GS_CUDA(cudaMemcpy(P->dPinv.p, pinv.data(), pinv.size() * 4, cudaMemcpyHostToDevice));
    if ((int)v.size() >= kMaxPatterns) v.erase(v.begin());
    v.push_back(std::move(P));
    *out = v.back().get();
    return GS_OK;
}

// Factorise and solve the `cnt` systems loaded into G's workspace (FP64): the fused factorisation + forward
// substitution level by level, then the backward substitution; the solution is left in y (pivot order).
int LinearSolve(gs_grid* G, int cnt) {
    using T = double;
    gs_ctx* ctx = G->ctx;
    const Symbolic& s = G->sym;
    const DevBatch b = MakeBatch(G, cnt, false);
    const DevGrid& g = G->view;
    cudaStream_t st = ctx->stream;
    const int grp = (cnt + Lay<T>::S - 1) / Lay<T>::S;
    const dim3 blk4(32, 4), blkP(32, kPersistWarps);
    auto level = [&](auto kernel, int i0, int i1) {
        if (i1 > i0) kernel<<<dim3((i1 - i0 + 3) / 4, grp), blk4, 0, st>>>(g, b, (T*)b.y, i0, i1);
    };
    const auto& fp = s.factor.levelItemPtr;
    const auto& bp = s.backward.levelItemPtr;
    const int split = G->split, splitB = G->splitB;  // the scalar schedule
    for (int l = 0; l < split; l++) {
        level(k_level<T, kWorkFactor>, fp[2 * l], fp[2 * l + 1]);
        level(k_level<T, kWorkFactor>, fp[2 * l + 1], fp[2 * l + 2]);
    }
    if (split < s.nLevels) k_persistent<T, kWorkFactor><<<grp, blkP, 0, st>>>(g, b, (T*)b.y, split, s.nLevels);
    if (splitB < s.nLevels) k_persistent<T, kWorkBackward><<<grp, blkP, 0, st>>>(g, b, (T*)b.y, splitB, s.nLevels);
    for (int l = splitB - 1; l >= 0; l--) level(k_level<T, kWorkBackward>, bp[l], bp[l + 1]);
    GS_CUDA(cudaGetLastError());
    return GS_OK;
}

}  // namespace
}  // namespace gs

extern "C" {

int gs_sparse_solve_batch(gs_ctx* ctx, int32_t count, const int32_t* n, const int32_t* rowPtr, const int32_t* colIdx,
                          const double* values, const double* rhs, double* x, int32_t* status) {
    if (!ctx || count < 0) return GS_ERR_INVALID_ARG;
    if (count == 0) return GS_OK;
    if (!n || !rowPtr || !colIdx || !values || !rhs || !x || !status) return GS_ERR_INVALID_ARG;
    // each system's blocks; a block whose size cannot be read makes the call malformed
    std::vector<int64_t> rpOff(count), nzOff(count), vOff(count);
    int64_t a = 0, z = 0, v = 0;
    for (int q = 0; q < count; q++) {
        if (n[q] <= 0) return SetErr(ctx, GS_ERR_INVALID_ARG, "system " + std::to_string(q) + " has no rows");
        rpOff[q] = a; nzOff[q] = z; vOff[q] = v;
        const int nnz = rowPtr[a + n[q]];
        if (nnz < 0) return SetErr(ctx, GS_ERR_INVALID_ARG, "system " + std::to_string(q) + " has a negative entry count");
        a += n[q] + 1; z += nnz; v += n[q];
    }
    GS_CUDA(cudaSetDevice(ctx->device));
    // per-system checks (ArgumentException per system in the reference), then systems grouped by pattern. A system
    // whose right-hand side is not finite is factorised all the same (with a zero right-hand side in its place), as
    // CpuSparseLuSolver factors before it checks b (PowerFlow/CpuSparseLuSolver.cs:41-47): singular if the
    // factorisation fails, else refused for its right-hand side; its x is never written.
    std::map<uint64_t, std::vector<int>> groups;
    std::vector<char> rhsBad(count, 0);
    for (int q = 0; q < count; q++) {
        const int nq = n[q];
        const int* rp = rowPtr + rpOff[q];
        const int* ci = colIdx + nzOff[q];
        bool ok = rp[0] == 0;
        for (int i = 0; i < nq && ok; i++) ok = rp[i + 1] >= rp[i];
        for (int i = 0; i < nq && ok; i++) {
            std::vector<int> row(ci + rp[i], ci + rp[i + 1]);
            std::sort(row.begin(), row.end());
            ok = (row.empty() || (row.front() >= 0 && row.back() < nq)) &&
                 std::adjacent_find(row.begin(), row.end()) == row.end();
        }
        if (!ok) { status[q] = GS_LS_MALFORMED; continue; }
        bool finite = true;
        for (int p = 0; p < rp[nq] && finite; p++) finite = std::isfinite(values[nzOff[q] + p]);
        if (!finite) { status[q] = GS_LS_NON_FINITE_INPUT; continue; }
        for (int i = 0; i < nq && !rhsBad[q]; i++) rhsBad[q] = !std::isfinite(rhs[vOff[q] + i]);
        status[q] = GS_LS_OK;
        groups[PatternHash(nq, rp, ci)].push_back(q);
    }
    gs_pf_opts o;
    gs_pf_opts_default(&o);
    for (auto& kv : groups) {
        // one hash may hold several patterns: split the list by exact pattern
        std::vector<int> todo = kv.second;
        while (!todo.empty()) {
            const int q0 = todo.front();
            const int nq = n[q0];
            const int* rp0 = rowPtr + rpOff[q0];
            const int* ci0 = colIdx + nzOff[q0];
            const int nnz = rp0[nq];
            std::vector<int> same, rest;
            for (int q : todo) {
                const bool eq = n[q] == nq && std::equal(rp0, rp0 + nq + 1, rowPtr + rpOff[q]) &&
                                std::equal(ci0, ci0 + nnz, colIdx + nzOff[q]);
                (eq ? same : rest).push_back(q);
            }
            todo.swap(rest);
            MatrixPattern* P = nullptr;
            int rc = PatternOf(ctx, nq, rp0, ci0, &P);
            if (rc) return rc;
            gs_grid* G = P->grid.get();
            int done = 0;
            while (done < (int)same.size()) {
                const int want = (int)same.size() - done;
                const int B = ChooseB(G, want, o);
                if ((rc = EnsureWorkspace(G, B, GS_PREC_FP64, false, false)) != GS_OK) return rc;
                const int cnt = std::min(B, want);
                std::vector<double> hv((size_t)cnt * nnz), hb((size_t)cnt * nq);
                for (int c = 0; c < cnt; c++) {
                    const int q = same[done + c];
                    std::copy(values + nzOff[q], values + nzOff[q] + nnz, hv.begin() + (size_t)c * nnz);
                    if (rhsBad[q]) std::fill(hb.begin() + (size_t)c * nq, hb.begin() + (size_t)(c + 1) * nq, 0.0);
                    else std::copy(rhs + vOff[q], rhs + vOff[q] + nq, hb.begin() + (size_t)c * nq);
                }
                DevBuf dv, db;
                GS_CUDA(dv.alloc(std::max<size_t>(8, hv.size() * 8)));
                GS_CUDA(db.alloc(hb.size() * 8));
                if (!hv.empty()) GS_CUDA(cudaMemcpy(dv.p, hv.data(), hv.size() * 8, cudaMemcpyHostToDevice));
                GS_CUDA(cudaMemcpy(db.p, hb.data(), hb.size() * 8, cudaMemcpyHostToDevice));
                const DevBatch b = MakeBatch(G, cnt, false);
                k_load_matrix<<<dim3((std::max(nnz, nq) + 7) / 8, B / 32), dim3(32, 8), 0, ctx->stream>>>(
                    b, cnt, nnz, nq, P->dSlot.as<int>(), P->dPinv.as<int>(), dv.as<double>(), db.as<double>());
                GS_CUDA(cudaGetLastError());
                if ((rc = LinearSolve(G, cnt)) != GS_OK) return rc;
                std::vector<double> y((size_t)nq * B);
                std::vector<int> fl(cnt);
                GS_CUDA(cudaMemcpyAsync(y.data(), G->ws.y.p, y.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
                GS_CUDA(cudaMemcpyAsync(fl.data(), G->ws.flags.p, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
                GS_CUDA(cudaStreamSynchronize(ctx->stream));
                const std::vector<int>& pinv = G->sym.pinv;
                std::vector<int> redo;  // systems whose static pivot collapsed (or whose solution is not finite)
                for (int c = 0; c < cnt; c++) {
                    const int q = same[done + c];
                    bool good = !(fl[c] & kFlagPivotPerturbed);
                    for (int i = 0; i < nq && good; i++) good = std::isfinite(y[(size_t)pinv[i] * B + c]);
                    if (!good) { redo.push_back(c); continue; }
                    if (rhsBad[q]) { status[q] = GS_LS_NON_FINITE_INPUT; continue; }
                    for (int i = 0; i < nq; i++) x[vOff[q] + i] = y[(size_t)pinv[i] * B + c];
                }
                if (!redo.empty()) {
                    // solved again with row partial pivoting (the reference's factorisation) from the reloaded
                    // matrix; singular only if that fails too
                    k_load_matrix<<<dim3((std::max(nnz, nq) + 7) / 8, B / 32), dim3(32, 8), 0, ctx->stream>>>(
                        b, cnt, nnz, nq, P->dSlot.as<int>(), P->dPinv.as<int>(), dv.as<double>(), db.as<double>());
                    DevBuf dl;
                    GS_CUDA(dl.alloc(redo.size() * 4));
                    GS_CUDA(cudaMemcpy(dl.p, redo.data(), redo.size() * 4, cudaMemcpyHostToDevice));
                    int gl = 0;
                    if ((rc = GpStep(G, b, dl.as<int>(), (int)redo.size(), ctx->stream, &gl)) != GS_OK) return rc;
                    GS_CUDA(cudaMemcpyAsync(y.data(), G->ws.y.p, y.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
                    GS_CUDA(cudaMemcpyAsync(fl.data(), G->ws.flags.p, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
                    GS_CUDA(cudaStreamSynchronize(ctx->stream));
                    for (int c : redo) {
                        const int q = same[done + c];
                        if (fl[c] & kFlagPivotFailed) { status[q] = GS_LS_SINGULAR; continue; }
                        if (rhsBad[q]) { status[q] = GS_LS_NON_FINITE_INPUT; continue; }
                        for (int i = 0; i < nq; i++) x[vOff[q] + i] = y[(size_t)pinv[i] * B + c];
                    }
                }
                done += cnt;
            }
        }
    }
    return GS_OK;
}

}  // extern "C"

// =============================================================================================
// Allocation-free mismatch evaluation.
//
// For callers that must not allocate device memory at the point where they check a state: a host whose device
// memory is all handed out up front by its own pool (a managed host that reserves its budget once, a process held
// to a fixed share of a GPU it shares with others), or a latency-bound control loop, where cudaMalloc / cudaFree
// may synchronise the whole device and stall its other streams. They hand in device arrays they already own; the
// only scratch this entry point needs (one max-norm accumulator and one flag word per system, 16 bytes) lives in
// the file-scope array below: 2 x 65,536 x 8 bytes = 1 MiB, which every GPU that loads this library holds until
// the process exits. Calls that overlap on the GPU share it and race: issue them one after another.
namespace gs {

constexpr int kNoAllocMaxSystems = 65536;

// [0, max): max |f| accumulators (bits of a non-negative double); [max, 2 max): non-finite flags (as words)
static __device__ __align__(256) unsigned long long gNoAllocScratch[2 * kNoAllocMaxSystems];

// Variant of k_mismatch_jac without the Jacobian fill: per (bus, system) the FP64 injections and the
// mismatch of this bus's equations, reduced to a per-system max |f| in the static scratch. Inputs are
// system-major ([count][n]); Va in radians; outage[s] removes one branch (or -1).
__global__ void __launch_bounds__(256) k_mismatch_noalloc(DevGrid g, int count, const double* __restrict__ vm,
                                                          const double* __restrict__ va, const int* __restrict__ outage,
                                                          unsigned long long* acc, unsigned long long* bad) {
    const int lane = threadIdx.x, w = threadIdx.y;
    const int s = blockIdx.y * 32 + lane;
    const int i = blockIdx.x * 8 + w;
    double localMax = 0.0;
    int nonFinite = 0;
    if (i < g.n && s < count) {
        const size_t row = (size_t)s * g.n;
        int o = outage ? outage[s] : -1;
        if (o >= g.nbr) { o = -1; nonFinite = 1; }  // not a branch of this grid: the result is NaN
        int c0 = -1, c1 = -1, c2 = -1, c3 = -1;
        if (o >= 0) { c0 = g.brCell[4 * o]; c1 = g.brCell[4 * o + 1]; c2 = g.brCell[4 * o + 2]; c3 = g.brCell[4 * o + 3]; }
        const double vmi = vm[row + i], vai = va[row + i];
        double pi = 0.0, qi = 0.0;
        for (int p = g.yRowPtr[i]; p < g.yRowPtr[i + 1]; p++) {
            const int j = g.yCol[p];
            double G = g.yG[p], Bv = g.yB[p];
            if (p == c0) { G = g.brRed[8 * o + 0]; Bv = g.brRed[8 * o + 1]; }
            else if (p == c1) { G = g.brRed[8 * o + 2]; Bv = g.brRed[8 * o + 3]; }
            else if (p == c2) { G = g.brRed[8 * o + 4]; Bv = g.brRed[8 * o + 5]; }
            else if (p == c3) { G = g.brRed[8 * o + 6]; Bv = g.brRed[8 * o + 7]; }
            double sn, cs;
            sincos(vai - va[row + j], &sn, &cs);
            const double vmj = vm[row + j];
            pi += vmj * (G * cs + Bv * sn);
            qi += vmj * (G * sn - Bv * cs);
        }
        const double P = vmi * pi, Q = vmi * qi;
        // a voltage-dependent (ZIP) load's deviation from its nominal power, as the solver's mismatch takes it
        double zdP = 0.0, zdQ = 0.0, zdPdV = 0.0, zdQdV = 0.0;
        zipLoad(g, i, vmi, g.pload[i], g.qload[i], zdP, zdQ, zdPdV, zdQdV);
        if (g.busP[i] >= 0) {
            const double f = (g.pgen[i] - g.pload[i]) - P - zdP;
            localMax = fmax(localMax, fabs(f));
            nonFinite |= isfinite(f) ? 0 : 1;
        }
        if (g.busQ[i] >= 0) {
            const double f = (g.qgen[i] - g.qload[i]) - Q - zdQ;
            localMax = fmax(localMax, fabs(f));
            nonFinite |= isfinite(f) ? 0 : 1;
        }
    }
    __shared__ double red[8][32];
    __shared__ int redBad[8][32];
    red[w][lane] = localMax;
    redBad[w][lane] = nonFinite;
    __syncthreads();
    if (w == 0 && s < count) {
        double mx = red[0][lane];
        int anyBad = redBad[0][lane];
        for (int q = 1; q < 8; q++) { mx = fmax(mx, red[q][lane]); anyBad |= redBad[q][lane]; }
        if (mx > 0.0) atomicMaxNonNeg(&acc[s], mx);
        if (anyBad) atomicOr(&bad[s], 1ull);
    }
}

__global__ void k_noalloc_clear(int count, unsigned long long* acc, unsigned long long* bad) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < count) { acc[s] = 0ull; bad[s] = 0ull; }
}

__global__ void k_noalloc_finish(int count, const unsigned long long* acc, const unsigned long long* bad, double* out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < count) out[s] = bad[s] ? NAN : __longlong_as_double((long long)acc[s]);
}

namespace {
std::mutex gNoAllocMu;  // guards the per-context lookup of the scratch array's device address
}  // namespace

}  // namespace gs

extern "C" int gs_pf_mismatch_noalloc(gs_grid* G, int32_t count, const double* d_vm, const double* d_va,
                                      const int32_t* d_outage, double* d_max_mismatch) {
    using namespace gs;
    if (!G || count < 0 || (count > 0 && (!d_vm || !d_va || !d_max_mismatch))) return GS_ERR_INVALID_ARG;
    gs_ctx* ctx = G->ctx;
    if (count > kNoAllocMaxSystems)
        return SetErr(ctx, GS_ERR_CAPACITY, "gs_pf_mismatch_noalloc: " + std::to_string(count) +
                                              " systems requested, at most " + std::to_string(kNoAllocMaxSystems));
    if (count == 0) return GS_OK;
    GS_CUDA(cudaSetDevice(ctx->device));
    unsigned long long* scratch = nullptr;
    {
        // On the context's first call, with its device current: the device address of the static scratch array.
        // The host-side name gNoAllocScratch is only a stand-in for it, never a device address. The address is
        // kept per context (not per device ordinal for the whole process): a context is created against the
        // device's current CUDA context, so a device reset, after which the module may load elsewhere, comes
        // with a new gs_ctx and a new lookup.
        std::lock_guard<std::mutex> lock(gNoAllocMu);
        if (!ctx->noallocScratch) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, gNoAllocScratch);
            if (e != cudaSuccess)
                return SetErr(ctx, GS_ERR_CUDA, std::string("cudaGetSymbolAddress(gNoAllocScratch): ") + cudaGetErrorString(e));
            ctx->noallocScratch = static_cast<unsigned long long*>(p);
        }
        scratch = ctx->noallocScratch;
    }
    unsigned long long* acc = scratch;
    unsigned long long* bad = scratch + kNoAllocMaxSystems;
    cudaStream_t st = ctx->stream;
    k_noalloc_clear<<<(count + 255) / 256, 256, 0, st>>>(count, acc, bad);
    k_mismatch_noalloc<<<dim3((G->sym.n + 7) / 8, (count + 31) / 32), dim3(32, 8), 0, st>>>(G->view, count, d_vm, d_va,
                                                                                           d_outage, acc, bad);
    k_noalloc_finish<<<(count + 255) / 256, 256, 0, st>>>(count, acc, bad, d_max_mismatch);
    GS_CUDA(cudaGetLastError());
    GS_CUDA(cudaStreamSynchronize(st));
    return GS_OK;
}

// The uneven multi-grid batch (gs_pf_solve_multi) and the request loop (gs_serve_*): they use the kernels and
// host helpers above.
#include "gs_multi.cuh"
#include "gs_serve.cuh"

namespace gs {
// the one-system kernels hold the top of the elimination tree in up to 200 KB of dynamic shared memory
cudaError_t SetKernelAttributes() {
    const int bytes = 220 * 1024;  // the 200 KB budget of the top part plus the walk counters
    cudaError_t e = cudaSuccess;
    auto set = [&](const void* f) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    };
    set((const void*)k_tail<float, kWorkFactor>);
    set((const void*)k_tail<float, kWorkBackward>);
    set((const void*)k_tail<float, kWorkForward>);
    set((const void*)k_tail<double, kWorkFactor>);
    set((const void*)k_tail<double, kWorkBackward>);
    set((const void*)k_tail<double, kWorkForward>);
    set((const void*)k_newton<float>);
    set((const void*)k_newton<double>);
    return e;
}
}  // namespace gs

namespace gs {
// Whether a cluster of kClusterCtas CTAs of the few-systems cluster walk fits on this device (checked per context).
bool ClusterWalkAvailable() {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClusterCtas);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = kClusterSmemMax;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
#define GS_CLUSTER_KERNELS(C, PK)                                                                                  \
    (const void*)k_tail_cluster<double, kWorkFactor, C, PK>, (const void*)k_tail_cluster<double, kWorkBackward, C, PK>, \
        (const void*)k_tail_cluster<double, kWorkForward, C, PK>, (const void*)k_tail_cluster<float, kWorkFactor, C, PK>, \
        (const void*)k_tail_cluster<float, kWorkBackward, C, PK>, (const void*)k_tail_cluster<float, kWorkForward, C, PK>
    for (const void* f : {GS_CLUSTER_KERNELS(1, false), GS_CLUSTER_KERNELS(2, false), GS_CLUSTER_KERNELS(4, false),
                          GS_CLUSTER_KERNELS(8, false), GS_CLUSTER_KERNELS(1, true), GS_CLUSTER_KERNELS(2, true),
                          GS_CLUSTER_KERNELS(4, true), GS_CLUSTER_KERNELS(8, true)})
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClusterSmemMax) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
#undef GS_CLUSTER_KERNELS
#define GS_CLUSTER_KERNELS16(PK)                                                                                   \
    (const void*)k_tail_cluster<double, kWorkFactor, 16, PK>, (const void*)k_tail_cluster<double, kWorkBackward, 16, PK>, \
        (const void*)k_tail_cluster<double, kWorkForward, 16, PK>, (const void*)k_tail_cluster<float, kWorkFactor, 16, PK>, \
        (const void*)k_tail_cluster<float, kWorkBackward, 16, PK>, (const void*)k_tail_cluster<float, kWorkForward, 16, PK>
    // the largest portable cluster must fit (the smaller ones then do)
    for (const void* f : {(const void*)k_tail_cluster<double, kWorkFactor, kClusterCtas, false>,
                          (const void*)k_tail_cluster<double, kWorkFactor, kClusterCtas, true>,
                          (const void*)k_tail_cluster<float, kWorkFactor, kClusterCtas, true>})
        if (cudaOccupancyMaxActiveClusters(&n, f, &cfg) != cudaSuccess || n < 1) {
            cudaGetLastError();
            return false;
        }
    // 16-CTA clusters (non-portable) for the last few systems, where the device schedules them
    bool ok16 = true;
    const void* k16[] = {GS_CLUSTER_KERNELS16(false), GS_CLUSTER_KERNELS16(true)};
    for (const void* f : k16)
        ok16 = ok16 && cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess &&
               cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClusterSmemMax) == cudaSuccess;
    if (ok16) {
        cfg.gridDim = dim3(kClusterCtasWide);
        attr[0].val.clusterDim.x = kClusterCtasWide;
        for (const void* f : k16)
            if (cudaOccupancyMaxActiveClusters(&n, f, &cfg) != cudaSuccess || n < 1) { ok16 = false; break; }
    }
#undef GS_CLUSTER_KERNELS16
    cudaGetLastError();
    Cluster16Ok() = ok16;
    return true;
}
}  // namespace gs
