// gs_paired.cuh — the factorisation and triangular solves on the paired schedule (Symbolic::PairSchedule), sm_100a.
//
// A PQ bus's angle and magnitude unknowns are eliminated one after the other with the same structure, so the two
// nodes k, k + 1 form one 2 x 2 block. Their entries are computed together: L(k + 1, j) sits one slot after L(k, j),
// U(j, k + 1) one after U(j, k), so one index pair stands for two (or, in the diagonal block, four) products, and the
// tree of units has about half the levels of the node tree (121 against 212 on the 10,000-bus grid, 0.87 M index
// pairs against 1.71 M). The LU storage is the node-major one of the scalar schedule, so every other kernel (the
// fill, the one-system walks, the residual) reads the same factors.
//
// Task descriptors: A = {first pair, end of pairs, kind | hasA bits << 3, node k}, B = {s0, s1, aux, 0} (see
// gs_internal.h). Products per index pair (a, c): K = 1 lu[a] R[c]; K = 2 (left pair) lu[a] R[c], lu[a + 1] R[c];
// K = 3 (right pair) lu[a] R[c], lu[a] R[c + 1]; K = 4 (block) the four products of lu[a .. a + 1] and R[c .. c + 1].
#pragma once

namespace gs {

__device__ __forceinline__ int pkKind(const int4& a) { return a.z & 7; }
__device__ __forceinline__ bool pkHasA(const int4& a, int i) { return (a.z >> (3 + i)) & 1; }
// products an index pair stands for, by task kind
__device__ __forceinline__ int pkProducts(int kind) {
    return kind == kPDiag ? 4 : kind == kPLower ? 3 : (kind == kPUpper || kind == kPFwd) ? 2 : 1;
}

// acc += the K products of pair (a, c) for system s (lu and R interleaved with stride B)
template <typename T, int K>
__device__ __forceinline__ void pkAcc(const T* lu, const T* R, int a, int c, size_t B, int s, T (&acc)[4]) {
    const T l0 = lu[(size_t)a * B + s];
    const T r0 = R[(size_t)c * B + s];
    if (K == 1) { acc[0] += l0 * r0; return; }
    if (K == 2) { const T l1 = lu[(size_t)(a + 1) * B + s]; acc[0] += l0 * r0; acc[1] += l1 * r0; return; }
    const T r1 = R[(size_t)(c + 1) * B + s];
    if (K == 3) { acc[0] += l0 * r0; acc[1] += l0 * r1; return; }
    const T l1 = lu[(size_t)(a + 1) * B + s];
    acc[0] += l0 * r0; acc[1] += l0 * r1; acc[2] += l1 * r0; acc[3] += l1 * r1;
}

// The sums of a task over pairs [q0, q1) for this lane's system, in the batched layout (S systems x P pair lanes).
// Warp mode: the warp's lanes load 32 pairs together, pair lane pl takes pairs pl, pl + P, ..., and a fixed butterfly
// over the pair lanes completes every sum in every lane. Thread mode: this lane alone, four pairs in flight.
template <typename T, int K>
__device__ __forceinline__ void pkSumWarp(const T* lu, const T* R, const int2* __restrict__ pr, int q0, int q1, size_t B,
                                          int s, T (&acc)[4]) {
    // pairs per round: four, two for FP64 with three or four products a pair (the level kernels' register budget)
    constexpr int S = Lay<T>::S, P = Lay<T>::P, U = (sizeof(T) == 8 && K >= 3) ? 2 : 4;
    const int lane = threadIdx.x & 31, pl = lane / S;
    for (int base = q0; base < q1; base += 32) {
        const int cnt = min(32, q1 - base);
        const int2 mine = lane < cnt ? __ldg(pr + base + lane) : make_int2(0, 0);
        // four pairs' operands loaded (predicated, not branched) before any product, so their loads are in flight
        // together
#pragma unroll
        for (int u0 = 0; u0 < S; u0 += U) {
            T l0[U], l1[U], r0[U], r1[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int src = pl + P * (u0 + u);
                const int a = __shfl_sync(0xffffffffu, mine.x, src);
                const int c = __shfl_sync(0xffffffffu, mine.y, src);
                const bool ok = src < cnt;
                l0[u] = ok ? lu[(size_t)a * B + s] : T(0);
                r0[u] = ok ? R[(size_t)c * B + s] : T(0);
                l1[u] = (ok && (K == 2 || K == 4)) ? lu[(size_t)(a + 1) * B + s] : T(0);
                r1[u] = (ok && (K == 3 || K == 4)) ? R[(size_t)(c + 1) * B + s] : T(0);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                acc[0] += l0[u] * r0[u];
                if (K == 2) acc[1] += l1[u] * r0[u];
                if (K == 3) acc[1] += l0[u] * r1[u];
                if (K == 4) { acc[1] += l0[u] * r1[u]; acc[2] += l1[u] * r0[u]; acc[3] += l1[u] * r1[u]; }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
        if (i < (K == 4 ? 4 : K == 1 ? 1 : 2))
#pragma unroll
            for (int off = S; off < 32; off <<= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
}

template <typename T, int K>
__device__ __forceinline__ void pkSumThread(const T* lu, const T* R, const int2* __restrict__ pr, int q0, int q1, size_t B,
                                            int s, T (&acc)[4]) {
    int q = q0;
    for (; q + 4 <= q1; q += 4) {
        const int2 p0 = __ldg(pr + q), p1 = __ldg(pr + q + 1), p2 = __ldg(pr + q + 2), p3 = __ldg(pr + q + 3);
        pkAcc<T, K>(lu, R, p0.x, p0.y, B, s, acc);
        pkAcc<T, K>(lu, R, p1.x, p1.y, B, s, acc);
        pkAcc<T, K>(lu, R, p2.x, p2.y, B, s, acc);
        pkAcc<T, K>(lu, R, p3.x, p3.y, B, s, acc);
    }
    for (; q < q1; q++) {
        const int2 p = __ldg(pr + q);
        pkAcc<T, K>(lu, R, p.x, p.y, B, s, acc);
    }
}

// How a task is shared: one lane per system alone (serial), the S lanes of a lane group (its S systems) with the
// index pairs loaded by the group together, or the whole warp (pair lanes).
enum PkMode { kPkThread = 0, kPkGroup = 1, kPkWarp = 2 };

// Group mode, for short tasks (at most 32 index pairs) in the latency-bound walks: the group's S lanes load all the
// pairs in one round (32 / S each), then every lane gathers its own system's operands in rounds of eight pairs that
// do not depend on each other: two dependent rounds of loads however long the task.
template <typename T, int K>
__device__ __forceinline__ void pkSumGroup(const T* lu, const T* R, const int2* __restrict__ pr, int q0, int q1,
                                           size_t B, int s, T (&acc)[4]) {
    constexpr int S = Lay<T>::S, KS = 32 / S, RK = 8 / S;  // pair slots per lane; slots per round of eight pairs
    const int lane = threadIdx.x & 31, gbase = lane & ~(S - 1), j = lane & (S - 1);
    const unsigned mask = ((1u << S) - 1u) << gbase;
    const int n = q1 - q0;
    int2 mine[KS];
#pragma unroll
    for (int k = 0; k < KS; k++) mine[k] = j + k * S < n ? __ldg(pr + q0 + j + k * S) : make_int2(0, 0);
#pragma unroll
    for (int k0 = 0; k0 < KS; k0 += RK) {
        if (k0 * S >= n) break;  // uniform over the group
        T l0[8], l1[8], r0[8], r1[8];
#pragma unroll
        for (int kk = 0; kk < RK; kk++)
#pragma unroll
            for (int jj = 0; jj < S; jj++) {
                const int u = kk * S + jj;
                const int a = __shfl_sync(mask, mine[k0 + kk].x, gbase + jj);
                const int c = __shfl_sync(mask, mine[k0 + kk].y, gbase + jj);
                const bool ok = (k0 + kk) * S + jj < n;
                l0[u] = ok ? lu[(size_t)a * B + s] : T(0);
                r0[u] = ok ? R[(size_t)c * B + s] : T(0);
                l1[u] = (ok && (K == 2 || K == 4)) ? lu[(size_t)(a + 1) * B + s] : T(0);
                r1[u] = (ok && (K == 3 || K == 4)) ? R[(size_t)(c + 1) * B + s] : T(0);
            }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            acc[0] += l0[u] * r0[u];
            if (K == 2) acc[1] += l1[u] * r0[u];
            if (K == 3) acc[1] += l0[u] * r1[u];
            if (K == 4) { acc[1] += l0[u] * r1[u]; acc[2] += l1[u] * r0[u]; acc[3] += l1[u] * r1[u]; }
        }
    }
}

template <typename T, int K, int M>
__device__ __forceinline__ void pkSum(const T* lu, const T* R, const int2* pr, int q0, int q1, size_t B, int s,
                                      T (&acc)[4]) {
    if (M == kPkWarp) pkSumWarp<T, K>(lu, R, pr, q0, q1, B, s, acc);
    else if (M == kPkGroup) pkSumGroup<T, K>(lu, R, pr, q0, q1, B, s, acc);
    else pkSumThread<T, K>(lu, R, pr, q0, q1, B, s, acc);
}

// the diagonal of a factorisation: a - dot, perturbed to the floor of |a| when it collapses (the system flagged)
template <typename T>
__device__ __forceinline__ T pkPivot(const DevBatch& b, int s, T a, T v, bool flag) {
    const T fl = pivotFloor<T>() * (fabs(a) > T(1) ? fabs(a) : T(1));
    if (!(fabs(v) > fl)) {
        if (flag) atomicOr(&b.flags[s], kFlagPivotPerturbed);
        v = (v < T(0)) ? -fl : fl;
    }
    return v;
}

// One task of the fused factorisation + forward substitution for this lane's system (WIDE: the whole warp, pair
// lanes; else this lane alone). The values a task combines with its sums (A, pivots, L(k + 1, k), U(k, k + 1)) are
// loaded before the sums, beside their operands.
template <typename T, int M>
__device__ __forceinline__ void pkFactorTask(const DevGrid& g, const DevBatch& b, const int4 A, const int4 D, int s,
                                             bool act) {
    constexpr bool WIDE = M == kPkWarp;
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    T* y = (T*)b.y;
    T* piv = (T*)b.piv;
    const int kind = pkKind(A), k = A.w;
    const bool writer = !WIDE || (threadIdx.x & 31) < Lay<T>::S;
    const bool flag = act && writer;
    const int2* pr = g.psPairs;
    auto at = [&](const T* p, int idx) { return p[(size_t)idx * B + s]; };
    auto put = [&](T* p, int idx, T v) { if (writer) p[(size_t)idx * B + s] = v; };
    T acc[4] = {T(0), T(0), T(0), T(0)};
    if (kind < 4) {  // a single node's entry (kDiag, kUpper, kFwd, kLower)
        const int slot = D.x;
        const T a = kind == kFwd ? at(y, slot) : (pkHasA(A, 0) ? at(lu, slot) : T(0));
        const T pv = kind == kLower ? at(piv, k) : T(1);
        pkSum<T, 1, M>(lu, kind == kFwd ? y : lu, pr, A.x, A.y, B, s, acc);
        T v = a - acc[0];
        if (kind == kDiag) { put(piv, k, pkPivot<T>(b, s, a, v, flag)); return; }
        if (kind == kLower) v = v / pv;
        put(kind == kFwd ? y : lu, slot, v);
        return;
    }
    if (kind == kPDiag) {  // the 2 x 2 diagonal block of k, k + 1
        const int bk = D.x, bk1 = D.y, c = D.z;
        const T a00 = pkHasA(A, 0) ? at(lu, bk) : T(0), a01 = pkHasA(A, 1) ? at(lu, bk + 1) : T(0);
        const T a10 = pkHasA(A, 2) ? at(lu, bk + 2 + c) : T(0), a11 = pkHasA(A, 3) ? at(lu, bk1) : T(0);
        pkSum<T, 4, M>(lu, lu, pr, A.x, A.y, B, s, acc);
        const T p0 = pkPivot<T>(b, s, a00, a00 - acc[0], flag);
        const T u01 = a01 - acc[1];
        const T l10 = (a10 - acc[2]) / p0;
        const T p1 = pkPivot<T>(b, s, a11, a11 - acc[3] - l10 * u01, flag);
        put(piv, k, p0);
        put(lu, bk + 1, u01);
        put(lu, bk + 2 + c, l10);
        put(piv, k + 1, p1);
        return;
    }
    if (kind == kPUpper) {  // U(k, r), U(k + 1, r)
        const T a0 = pkHasA(A, 0) ? at(lu, D.x) : T(0), a1 = pkHasA(A, 1) ? at(lu, D.y) : T(0);
        const T l10 = at(lu, D.z);
        pkSum<T, 2, M>(lu, lu, pr, A.x, A.y, B, s, acc);
        const T v0 = a0 - acc[0];
        put(lu, D.x, v0);
        put(lu, D.y, a1 - acc[1] - l10 * v0);
        return;
    }
    if (kind == kPLower) {  // L(r, k), L(r, k + 1)
        const T a0 = pkHasA(A, 0) ? at(lu, D.x) : T(0), a1 = pkHasA(A, 1) ? at(lu, D.y) : T(0);
        const T u01 = at(lu, D.z), p0 = at(piv, k), p1 = at(piv, k + 1);
        pkSum<T, 3, M>(lu, lu, pr, A.x, A.y, B, s, acc);
        const T v0 = (a0 - acc[0]) / p0;
        put(lu, D.x, v0);
        put(lu, D.y, (a1 - acc[1] - v0 * u01) / p1);
        return;
    }
    {  // kPFwd: y(k), y(k + 1)
        const T y0 = at(y, k), y1 = at(y, k + 1), l10 = at(lu, D.z);
        pkSum<T, 2, M>(lu, y, pr, A.x, A.y, B, s, acc);
        const T v0 = y0 - acc[0];
        put(y, k, v0);
        put(y, k + 1, y1 - acc[1] - l10 * v0);
    }
}

// forward substitution of a second right-hand side v (the refinement): a single node's forward entry, or a pair's
template <typename T, int M>
__device__ __forceinline__ void pkForwardTask(const DevGrid& g, const DevBatch& b, T* v, const int4 A, const int4 D, int s) {
    constexpr bool WIDE = M == kPkWarp;
    const size_t B = (size_t)b.B;
    const T* lu = (const T*)b.lu;
    const bool writer = !WIDE || (threadIdx.x & 31) < Lay<T>::S;
    T acc[4] = {T(0), T(0), T(0), T(0)};
    if (pkKind(A) == kFwd) {
        const T a = v[(size_t)D.x * B + s];
        pkSum<T, 1, M>(lu, v, g.psPairs, A.x, A.y, B, s, acc);
        if (writer) v[(size_t)D.x * B + s] = a - acc[0];
        return;
    }
    const int k = A.w;
    const T y0 = v[(size_t)k * B + s], y1 = v[(size_t)(k + 1) * B + s], l10 = lu[(size_t)D.z * B + s];
    pkSum<T, 2, M>(lu, v, g.psPairs, A.x, A.y, B, s, acc);
    const T v0 = y0 - acc[0];
    if (writer) {
        v[(size_t)k * B + s] = v0;
        v[(size_t)(k + 1) * B + s] = y1 - acc[1] - l10 * v0;
    }
}

// backward substitution of a unit: x(k) over U(k, r) from s0 + 1 (a single node), or x(k + 1) then x(k) over
// U(k + 1, r) from s1 and U(k, r) from s0, with U(k, k + 1) at aux (a pair); r over pRows[A.x .. A.y)
template <typename T, int M>
__device__ __forceinline__ void pkBackTask(const DevGrid& g, const DevBatch& b, T* x, const int4 A, const int4 D, int s) {
    constexpr bool WIDE = M == kPkWarp;
    constexpr int S = Lay<T>::S, P = Lay<T>::P;
    const size_t B = (size_t)b.B;
    const T* lu = (const T*)b.lu;
    const T* piv = (const T*)b.piv;
    const int k = A.w, c = A.y - A.x;
    const int* rows = g.pRows + A.x;
    const bool pair = A.z == kBPair;
    const int s0 = pair ? D.x : D.x + 1, s1 = D.y;
    const T x0 = x[(size_t)k * B + s], pk0 = piv[(size_t)k * B + s];
    const T x1 = pair ? x[(size_t)(k + 1) * B + s] : T(0), pk1 = pair ? piv[(size_t)(k + 1) * B + s] : T(1);
    const T u01 = pair ? lu[(size_t)D.z * B + s] : T(0);
    T a0 = T(0), a1 = T(0);
    if (WIDE) {
        const int lane = threadIdx.x & 31, pl = lane / S;
        for (int t0 = 0; t0 < c; t0 += 32) {
            const int cnt = min(32, c - t0);
            const int mine = lane < cnt ? __ldg(rows + t0 + lane) : 0;
            for (int u = 0; u < S; u++) {
                const int src = pl + P * u;
                const int r = __shfl_sync(0xffffffffu, mine, src);
                if (src < cnt) {
                    const T xr = x[(size_t)r * B + s];
                    a0 += lu[(size_t)(s0 + t0 + src) * B + s] * xr;
                    if (pair) a1 += lu[(size_t)(s1 + t0 + src) * B + s] * xr;
                }
            }
        }
#pragma unroll
        for (int off = S; off < 32; off <<= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, off);
            a1 += __shfl_xor_sync(0xffffffffu, a1, off);
        }
    } else if (M == kPkGroup) {  // at most 32 rows: the group loads them together, then every operand at once
        constexpr int KS = 32 / S, RK = 8 / S;
        const int lane = threadIdx.x & 31, gbase = lane & ~(S - 1), j = lane & (S - 1);
        const unsigned mask = ((1u << S) - 1u) << gbase;
        int mine[KS];
#pragma unroll
        for (int kk = 0; kk < KS; kk++) mine[kk] = j + kk * S < c ? __ldg(rows + j + kk * S) : 0;
#pragma unroll
        for (int k0 = 0; k0 < KS; k0 += RK) {
            if (k0 * S >= c) break;  // uniform over the group
            T xr[8], u0[8], u1[8];
#pragma unroll
            for (int kk = 0; kk < RK; kk++)
#pragma unroll
                for (int jj = 0; jj < S; jj++) {
                    const int u = kk * S + jj, t = (k0 + kk) * S + jj;
                    const int r = __shfl_sync(mask, mine[k0 + kk], gbase + jj);
                    const bool ok = t < c;
                    xr[u] = ok ? x[(size_t)r * B + s] : T(0);
                    u0[u] = ok ? lu[(size_t)(s0 + t) * B + s] : T(0);
                    u1[u] = (ok && pair) ? lu[(size_t)(s1 + t) * B + s] : T(0);
                }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                a0 += u0[u] * xr[u];
                a1 += u1[u] * xr[u];
            }
        }
    } else {
        for (int t = 0; t < c; t++) {
            const T xr = x[(size_t)__ldg(rows + t) * B + s];
            a0 += lu[(size_t)(s0 + t) * B + s] * xr;
            if (pair) a1 += lu[(size_t)(s1 + t) * B + s] * xr;
        }
    }
    if (!WIDE || (threadIdx.x & 31) < S) {
        if (!pair) { x[(size_t)k * B + s] = (x0 - a0) / pk0; return; }
        const T v1 = (x1 - a1) / pk1;
        x[(size_t)(k + 1) * B + s] = v1;
        x[(size_t)k * B + s] = (x0 - u01 * v1 - a0) / pk0;
    }
}

// One work item of the paired schedule W: a wide task by the whole warp, or up to `count` short tasks over the lane
// groups (the batched layout), each by its group in mode SHORT (serial lanes in the wide level launches, where many
// warps hide the latency; group loads in the latency-bound persistent walks).
template <typename T, int W, int SHORT>
__device__ __forceinline__ void pkDoItem(const DevGrid& g, const DevBatch& b, T* vec, int it, int s, bool act) {
    const int* items = W == kWorkFactor ? g.pfItems : (W == kWorkBackward ? g.pbItems : g.pvItems);
    const int4* da = W == kWorkFactor ? g.pfA : (W == kWorkBackward ? g.pbA : g.pvA);
    const int4* db = W == kWorkFactor ? g.pfB : (W == kWorkBackward ? g.pbB : g.pvB);
    const int start = __ldg(items + 2 * it), count = __ldg(items + 2 * it + 1);
    auto run = [&](int pos, auto modeTag) {
        constexpr int MD = decltype(modeTag)::value;
        const int4 A = __ldg(da + pos), D = __ldg(db + pos);
        if (W == kWorkFactor) pkFactorTask<T, MD>(g, b, A, D, s, act);
        else if (W == kWorkBackward) pkBackTask<T, MD>(g, b, vec, A, D, s);
        else pkForwardTask<T, MD>(g, b, vec, A, D, s);
    };
    if (count < 0) run(start, std::integral_constant<int, kPkWarp>{});
    else
        for (int p = (threadIdx.x & 31) / Lay<T>::S; p < count; p += Lay<T>::P)
            run(start + p, std::integral_constant<int, SHORT>{});
}

// One level (or phase) of the paired schedule, items [i0, i1): block (32, 4), a warp per item, S systems per warp.
template <typename T, int W>
__global__ void __launch_bounds__(128, 10) k_plevel(DevGrid g, DevBatch b, T* vec, int i0, int i1) {
    const int it = i0 + blockIdx.x * 4 + threadIdx.y;
    const int s = laneSystem<T>(blockIdx.y);
    if (it >= i1) return;
    bool act = s < b.count && b.active[s];
    if (W != kWorkFactor && vec != (T*)b.y) act = act && b.refine[s];
    if (!__any_sync(0xffffffffu, act)) return;
    pkDoItem<T, W, kPkThread>(g, b, vec, it, s, act);
}

// The subtrees below the subtree cut (BuildSubtrees): one CTA per (system group, subtree) factors its subtree alone,
// its stages bottom-up with block barriers. A subtree's
// tasks read only its own entries, which its CTA has just written: they come back from L1 / L2 instead of DRAM, which
// the per-level launches over the whole batch cannot give. Grid (system groups, subtrees): the largest subtrees of
// every group start first.
template <typename T>
__global__ void __launch_bounds__(128) k_psubtree(DevGrid g, DevBatch b, const int* __restrict__ subStage,
                                                 const int* __restrict__ stagePtr, const int* __restrict__ work) {
    const int s = laneSystem<T>(blockIdx.x);
    const bool act = s < b.count && b.active[s];
    if (!__syncthreads_or(act)) return;
    constexpr int S = Lay<T>::S, P = Lay<T>::P;
    const int lane = threadIdx.x & 31, grp = lane / S;
    const unsigned full = 0xffffffffu;
    const int q0 = __ldg(subStage + blockIdx.y), q1 = __ldg(subStage + blockIdx.y + 1);
    for (int q = q0; q < q1; q++) {
        const int w0 = __ldg(stagePtr + q), w1 = __ldg(stagePtr + q + 1);
        // a warp takes P tasks at a time: a short one (at most 32 pairs) by one lane group serially, as the level
        // kernels run short tasks; a long one by the whole warp (pair lanes)
        for (int base = w0 + threadIdx.y * P; base < w1; base += blockDim.y * P) {
            const int w = base + grp;
            const bool have = w < w1;
            int4 A = make_int4(0, 0, 0, 0), D = A;
            if (have) {
                const int pos = __ldg(work + w);  // the task's position in the factorisation's descriptor arrays
                A = __ldg(g.pfA + pos);
                D = __ldg(g.pfB + pos);
            }
            const bool wide = have && A.y - A.x > 32;
            if (have && !wide) pkFactorTask<T, kPkThread>(g, b, A, D, s, act);
            for (int j = 0; j < P; j++) {
                if (!__shfl_sync(full, (int)wide, j * S)) continue;
                const int4 Aw = make_int4(__shfl_sync(full, A.x, j * S), __shfl_sync(full, A.y, j * S),
                                          __shfl_sync(full, A.z, j * S), __shfl_sync(full, A.w, j * S));
                const int4 Dw = make_int4(__shfl_sync(full, D.x, j * S), __shfl_sync(full, D.y, j * S),
                                          __shfl_sync(full, D.z, j * S), __shfl_sync(full, D.w, j * S));
                pkFactorTask<T, kPkWarp>(g, b, Aw, Dw, s, act);
            }
        }
        __syncthreads();
    }
}

// The narrow top of the unit tree: one CTA per system group walks its levels [l0, l1) with block barriers.
template <typename T, int W>
__global__ void __launch_bounds__(32 * kPersistWarps) k_ppersistent(DevGrid g, DevBatch b, T* vec, int l0, int l1) {
    const int s = laneSystem<T>(blockIdx.x);
    bool act = s < b.count && b.active[s];
    if (W != kWorkFactor && vec != (T*)b.y) act = act && b.refine[s];
    if (!__syncthreads_or(act)) return;
    const int* ptr = W == kWorkFactor ? g.pfLevelPtr : (W == kWorkBackward ? g.pbLevelPtr : g.pvLevelPtr);
    const int phases = W == kWorkFactor ? 2 : 1;
    for (int step = 0; step < l1 - l0; step++) {
        const int l = W == kWorkBackward ? l1 - 1 - step : l0 + step;
        for (int ph = 0; ph < phases; ph++) {
            const int i0 = ptr[phases * l + ph], i1 = ptr[phases * l + ph + 1];
            for (int it = i0 + threadIdx.y; it < i1; it += blockDim.y) pkDoItem<T, W, kPkGroup>(g, b, vec, it, s, act);
            __syncthreads();
        }
    }
}

}  // namespace gs
