// gs_cluster.cuh — the few-systems path on thread-block clusters (sm_100a).
//
// When only a handful of systems are still stepping (the outages that never converge run to the iteration cap, as in
// the reference), the walk over the elimination-tree levels is pure latency: a level's piece costs a chain of
// dependent loads (descriptor, index pairs, operands, the value it updates, the pivot) and every warp waits for the
// slowest piece at the level barrier. Here every listed system gets a cluster of kClusterCtas CTAs: each level (and
// phase) of a schedule is dealt out over all warps of the cluster, and
//   * the static part of the chain (the next level's descriptors and first index pairs, which never change) is
//     loaded between the cluster barrier's arrive and wait, behind the other CTAs' work, and
//   * the value a piece updates and its pivot are loaded beside its first operands,
// so after the barrier a piece costs one round of operand loads. The walk covers every level, so the per-level
// launches of the wide bottom levels go away too.
//
// Coherence: the CTAs of a cluster run on different SMs, whose L1 caches do not see each other's stores, so every
// value another CTA may have written during the walk (LU entries, pivots, right-hand sides) is read with
// ld.global.cg (L2) and written with st.global.cg; barrier.cluster.arrive.release / wait.acquire orders those stores
// before the next level's loads. Index data is read through the read-only path.
//
// The work of a level is dealt statically: wide pieces to warps, mid-length pieces to 8-lane groups, short pieces to
// threads, round-robin over the cluster. Each piece is summed in the same lane order as the one-CTA walk (k_tail).
#pragma once

namespace gs {

constexpr int kClusterCtas = 8;        // the largest portable cluster: CTAs per system
constexpr int kClusterCtasWide = 16;   // the non-portable cluster size sm_100a allows, where the device takes it
constexpr int kClusterThreads = 512;   // threads per CTA (one CTA per SM at the walk's register count)
constexpr int kClusterMaxSystems = 296; // more systems than this: the full-batch step
// whether 16-CTA clusters of the walk can be scheduled (set once with the kernels' attributes)
inline bool& Cluster16Ok() {
    static bool ok = false;
    return ok;
}
// CTAs per system for n systems: as many as keep the systems' clusters within about one wave of the 148 SMs
inline int ClusterCtasFor(int n) {
    if (n <= 9 && Cluster16Ok()) return kClusterCtasWide;
    return n <= 18 ? 8 : n <= 37 ? 4 : n <= 74 ? 2 : 1;
}
constexpr size_t kClusterSmemMax = 64 * 1024;  // the per-phase table in shared memory (16 bytes a phase)

template <typename T>
__device__ __forceinline__ T ldL2(const T* p) { return __ldcg(p); }
template <typename T>
__device__ __forceinline__ void stL2(T* p, T v) { __stcg(p, v); }

// Pairs a lane keeps in flight per round: 256 for a warp-wide piece, 64 for an 8-lane group, 8 for a thread, which
// covers every piece of the benchmark grids in one round (the longest has 245 pairs; short pieces have at most 8).
constexpr int kClusterInFlight = 8;

// A phase's work cut into warp-sized units: unit u < nw is wide piece u (the whole warp), the next ceil(nm / 4) units
// hold four mid-length pieces each (one per 8-lane group), the rest 32 short pieces each (one per lane). Warp w of the
// cluster takes units w, w + (warps of the cluster), ...; with at most that many units a warp has one class of work per
// phase. Returns the schedule position of this lane's piece in unit u (-1: none) and its class (0, 1, 2 = G 32, 8, 1).
__device__ __forceinline__ int unitPiece(const int4 P, int u, int lane, int& cls) {
    const int nw = P.y, nm = P.z, nr = P.w - P.x - P.y - P.z, m4 = (nm + 3) >> 2;
    if (u < nw) { cls = 0; return P.x + u; }
    if (u < nw + m4) {
        cls = 1;
        const int p = 4 * (u - nw) + (lane >> 3);
        return p < nm ? P.x + nw + p : -1;
    }
    cls = 2;
    const int p = 32 * (u - nw - m4) + lane;
    return p < nr ? P.x + nw + nm + p : -1;
}
__device__ __forceinline__ int unitCount(const int4 P) {
    const int nw = P.y, nm = P.z, nr = P.w - P.x - P.y - P.z;
    return nw + ((nm + 3) >> 2) + ((nr + 31) >> 5);
}

// This lane's first round of index pairs of piece d for a group of G lanes: (LU slot, right-hand-side index) for
// factorisation and forward entries, (U slot, row) for a backward node; x = -1 past the end.
template <int W, int G, int UF>
__device__ __forceinline__ void clPairs(const DevGrid& g, const int4 d, int2 (&a)[UF]) {
    const int j = G == 1 ? 0 : (int)(threadIdx.x & (G - 1));
    if (W == kWorkBackward) {
        const int c = d.z, base = d.y;  // LU slots fit 32 bits (checked by the symbolic analysis)
        const int* rows = g.pRows + d.w;
#pragma unroll
        for (int u = 0; u < kClusterInFlight; u++) {
            const int t = j + u * G;
            a[u] = t < c ? make_int2(base + 1 + t, __ldg(rows + t)) : make_int2(-1, -1);
        }
    } else {
#pragma unroll
        for (int u = 0; u < kClusterInFlight; u++) {
            const int q = d.y + j + u * G;
            a[u] = q < d.z ? __ldg(g.pairs + q) : make_int2(-1, -1);
        }
    }
}
template <int W, int UF>
__device__ __forceinline__ void clPairsOf(const DevGrid& g, int cls, const int4 d, int2 (&a)[UF]) {
    if (cls == 0) clPairs<W, 32, UF>(g, d, a);
    else if (cls == 1) clPairs<W, 8, UF>(g, d, a);
    else clPairs<W, 1, UF>(g, d, a);
}

// One piece by a group of G lanes (G = 32, 8 or 1) from its loaded first round; the group's first lane writes. Lane j
// of the group takes pairs j, j + G, ..., kClusterInFlight in flight per round, then a fixed butterfly over the group.
template <typename T, int W, int G, int UF>
__device__ __forceinline__ void clRun(const DevGrid& g, const DevBatch& b, T* vec, const int4 d,
                                      const int2 (&a0)[UF], int s, unsigned mask) {
    constexpr int U = UF;
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    T* piv = (T*)b.piv;
    const int j = G == 1 ? 0 : (int)(threadIdx.x & (G - 1));
    const bool lead = j == 0;
    // where the result goes and what it combines with, loaded beside the first operands
    T* out;
    const T* rhs;
    T base = T(0), div = T(1);
    int kind = kUpper;
    if (W == kWorkBackward) {
        out = vec + (size_t)d.x * B + s;
        rhs = vec;
        if (lead) { base = ldL2(out); div = ldL2(piv + (size_t)d.x * B + s); }
    } else if (W == kWorkForward) {
        out = vec + (size_t)descNode(d) * B + s;
        rhs = vec;
        if (lead) base = ldL2(out);
    } else {
        kind = descKind(d);
        const int node = descNode(d);
        T* y = (T*)b.y;
        rhs = kind == kFwd ? y : lu;
        out = kind == kFwd ? y + (size_t)d.x * B + s
                           : (kind == kDiag ? piv + (size_t)node * B + s : lu + (size_t)d.x * B + s);
        if (lead) {
            if (kind == kFwd) base = ldL2(out);
            else if (descHasA(d)) base = ldL2(lu + (size_t)d.x * B + s);
            if (kind == kLower) div = ldL2(piv + (size_t)node * B + s);
        }
    }
    T acc = T(0);
    {
        T l[U], r[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool ok = a0[u].x >= 0;
            l[u] = ok ? ldL2(lu + (size_t)a0[u].x * B + s) : T(0);
            r[u] = ok ? ldL2(rhs + (size_t)a0[u].y * B + s) : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) acc += l[u] * r[u];
    }
    // further rounds (pieces longer than U G pairs)
    const int len = W == kWorkBackward ? d.z : d.z - d.y;
    for (int off = U * G; off < len; off += U * G) {
        int2 a[U];
        if (W == kWorkBackward) {
            const int* rows = g.pRows + d.w;
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = off + j + u * G;
                a[u] = t < len ? make_int2(d.y + 1 + t, __ldg(rows + t)) : make_int2(-1, -1);
            }
        } else {
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int q = d.y + off + j + u * G;
                a[u] = q < d.z ? __ldg(g.pairs + q) : make_int2(-1, -1);
            }
        }
        T l[U], r[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool ok = a[u].x >= 0;
            l[u] = ok ? ldL2(lu + (size_t)a[u].x * B + s) : T(0);
            r[u] = ok ? ldL2(rhs + (size_t)a[u].y * B + s) : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) acc += l[u] * r[u];
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(mask, acc, o);
    if (!lead) return;
    if (W == kWorkBackward) { stL2(out, (base - acc) / div); return; }
    T v = base - acc;
    if (W == kWorkFactor && kind == kDiag) {
        const T a = base;
        const T fl = pivotFloor<T>() * (fabs(a) > T(1) ? fabs(a) : T(1));
        if (!(fabs(v) > fl)) { atomicOr(&b.flags[s], kFlagPivotPerturbed); v = (v < T(0)) ? -fl : fl; }
    }
    if (W == kWorkFactor && kind == kLower) v = v / div;
    stL2(out, v);
}

// ---- the same walk on the paired schedule (gs_paired.cuh): a task's descriptors A, D and its index pairs ----

// This lane's first round of a paired task's index pairs: (a, c) of a factorisation or forward task, (t, row) of a
// backward task (row r = pRows[A.x + t]); x = -1 past the end.
template <int W, int G, int UF>
__device__ __forceinline__ void clPairsP(const DevGrid& g, const int4 A, int2 (&a)[UF]) {
    const int j = G == 1 ? 0 : (int)(threadIdx.x & (G - 1));
    if (W == kWorkBackward) {
        const int c = A.y - A.x;
        const int* rows = g.pRows + A.x;
#pragma unroll
        for (int u = 0; u < kClusterInFlight; u++) {
            const int t = j + u * G;
            a[u] = t < c ? make_int2(t, __ldg(rows + t)) : make_int2(-1, -1);
        }
    } else {
#pragma unroll
        for (int u = 0; u < kClusterInFlight; u++) {
            const int q = A.x + j + u * G;
            a[u] = q < A.y ? __ldg(g.psPairs + q) : make_int2(-1, -1);
        }
    }
}
template <int W, int UF>
__device__ __forceinline__ void clPairsPOf(const DevGrid& g, int cls, const int4 A, int2 (&a)[UF]) {
    if (cls == 0) clPairsP<W, 32, UF>(g, A, a);
    else if (cls == 1) clPairsP<W, 8, UF>(g, A, a);
    else clPairsP<W, 1, UF>(g, A, a);
}

// The K products of a round of U index pairs of a paired task, added to acc: every operand of the round is loaded
// (predicated, not branched) before the first product, so the round's loads are in flight together. Backward pairs
// are (t, row): U(k, r) from s0 + t, U(k + 1, r) from s1 + t, times x(r).
template <typename T, int W, int K, int UF>
__device__ __forceinline__ void clRoundP(const T* lu, const T* R, int s0, int s1, const int2 (&p)[UF],
                                         size_t B, int s, T (&acc)[4]) {
    constexpr int U = UF;
    T l0[U], l1[U], r0[U], r1[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const bool ok = p[u].x >= 0;
        if (W == kWorkBackward) {
            r0[u] = ok ? ldL2(R + (size_t)p[u].y * B + s) : T(0);
            l0[u] = ok ? ldL2(lu + (size_t)(s0 + p[u].x) * B + s) : T(0);
            l1[u] = (ok && K == 2) ? ldL2(lu + (size_t)(s1 + p[u].x) * B + s) : T(0);
            r1[u] = T(0);
        } else {
            l0[u] = ok ? ldL2(lu + (size_t)p[u].x * B + s) : T(0);
            r0[u] = ok ? ldL2(R + (size_t)p[u].y * B + s) : T(0);
            l1[u] = (ok && (K == 2 || K == 4)) ? ldL2(lu + (size_t)(p[u].x + 1) * B + s) : T(0);
            r1[u] = (ok && (K == 3 || K == 4)) ? ldL2(R + (size_t)(p[u].y + 1) * B + s) : T(0);
        }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
        acc[0] += l0[u] * r0[u];
        if (W == kWorkBackward) { if (K == 2) acc[1] += l1[u] * r0[u]; continue; }
        if (K == 2) acc[1] += l1[u] * r0[u];
        if (K == 3) acc[1] += l0[u] * r1[u];
        if (K == 4) { acc[1] += l0[u] * r1[u]; acc[2] += l1[u] * r0[u]; acc[3] += l1[u] * r1[u]; }
    }
}
template <typename T, int W, int UF>
__device__ __forceinline__ void clRoundPK(int K, const T* lu, const T* R, int s0, int s1, const int2 (&p)[UF],
                                          size_t B, int s, T (&acc)[4]) {
    if (K == 1) clRoundP<T, W, 1, UF>(lu, R, s0, s1, p, B, s, acc);
    else if (K == 2) clRoundP<T, W, 2, UF>(lu, R, s0, s1, p, B, s, acc);
    else if (K == 3) clRoundP<T, W, 3, UF>(lu, R, s0, s1, p, B, s, acc);
    else clRoundP<T, W, 4, UF>(lu, R, s0, s1, p, B, s, acc);
}

// One paired task by a group of G lanes from its loaded first round; the group's first lane writes its outputs.
template <typename T, int W, int G, int UF>
__device__ __forceinline__ void clRunP(const DevGrid& g, const DevBatch& b, T* vec, const int4 A, const int4 D,
                                       const int2 (&a0)[UF], int s, unsigned mask) {
    constexpr int U = UF;
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    T* piv = (T*)b.piv;
    T* y = (T*)b.y;
    const int j = G == 1 ? 0 : (int)(threadIdx.x & (G - 1));
    const bool lead = j == 0;
    const int k = A.w;
    const int kind = W == kWorkBackward ? A.z : pkKind(A);
    const int K = W == kWorkBackward ? (kind == kBPair ? 2 : 1) : pkProducts(kind);
    const T* R = W == kWorkFactor ? ((kind == kFwd || kind == kPFwd) ? y : lu) : vec;
    const int s0 = W == kWorkBackward ? (kind == kBPair ? D.x : D.x + 1) : 0, s1 = D.y;
    auto at = [&](const T* p, int idx) { return ldL2(p + (size_t)idx * B + s); };
    // the values the task's outputs combine with, loaded beside the first operands
    T e[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    if (lead) {
        if (W == kWorkBackward) {
            e[0] = at(vec, k); e[1] = at(piv, k);
            if (kind == kBPair) { e[2] = at(vec, k + 1); e[3] = at(piv, k + 1); e[4] = at(lu, D.z); }
        } else if (kind == kFwd) {
            e[0] = at(W == kWorkFactor ? y : vec, D.x);
        } else if (kind == kPFwd) {
            const T* v = W == kWorkFactor ? y : vec;
            e[0] = at(v, k); e[1] = at(v, k + 1); e[2] = at(lu, D.z);
        } else if (kind < 4) {
            e[0] = pkHasA(A, 0) ? at(lu, D.x) : T(0);
            if (kind == kLower) e[1] = at(piv, k);
        } else if (kind == kPDiag) {
            const int c = D.z;
            e[0] = pkHasA(A, 0) ? at(lu, D.x) : T(0);
            e[1] = pkHasA(A, 1) ? at(lu, D.x + 1) : T(0);
            e[2] = pkHasA(A, 2) ? at(lu, D.x + 2 + c) : T(0);
            e[3] = pkHasA(A, 3) ? at(lu, D.y) : T(0);
        } else {  // kPUpper (aux L(k + 1, k)) or kPLower (aux U(k, k + 1) and the two pivots)
            e[0] = pkHasA(A, 0) ? at(lu, D.x) : T(0);
            e[1] = pkHasA(A, 1) ? at(lu, D.y) : T(0);
            e[2] = at(lu, D.z);
            if (kind == kPLower) { e[3] = at(piv, k); e[4] = at(piv, k + 1); }
        }
    }
    T acc[4] = {T(0), T(0), T(0), T(0)};
    clRoundPK<T, W, UF>(K, lu, R, s0, s1, a0, B, s, acc);
    const int len = A.y - A.x;
    for (int off = U * G; off < len; off += U * G) {
        int2 a[U];
        if (W == kWorkBackward) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int t = off + j + u * G;
                a[u] = t < len ? make_int2(t, __ldg(g.pRows + A.x + t)) : make_int2(-1, -1);
            }
        } else {
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int q = A.x + off + j + u * G;
                a[u] = q < A.y ? __ldg(g.psPairs + q) : make_int2(-1, -1);
            }
        }
        clRoundPK<T, W, UF>(K, lu, R, s0, s1, a, B, s, acc);
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(mask, acc[i], o);
    if (!lead) return;
    auto put = [&](T* p, int idx, T v) { stL2(p + (size_t)idx * B + s, v); };
    if (W == kWorkBackward) {
        if (kind == kBNode) { put(vec, k, (e[0] - acc[0]) / e[1]); return; }
        const T v1 = (e[2] - acc[1]) / e[3];
        put(vec, k + 1, v1);
        put(vec, k, (e[0] - e[4] * v1 - acc[0]) / e[1]);
        return;
    }
    if (kind == kFwd) { put(W == kWorkFactor ? y : vec, D.x, e[0] - acc[0]); return; }
    if (kind == kPFwd) {
        T* v = W == kWorkFactor ? y : vec;
        const T v0 = e[0] - acc[0];
        put(v, k, v0);
        put(v, k + 1, e[1] - acc[1] - e[2] * v0);
        return;
    }
    if (kind < 4) {  // kDiag, kUpper, kLower
        T v = e[0] - acc[0];
        if (kind == kDiag) { put(piv, k, pkPivot<T>(b, s, e[0], v, true)); return; }
        if (kind == kLower) v = v / e[1];
        put(lu, D.x, v);
        return;
    }
    if (kind == kPDiag) {
        const T p0 = pkPivot<T>(b, s, e[0], e[0] - acc[0], true);
        const T u01 = e[1] - acc[1];
        const T l10 = (e[2] - acc[2]) / p0;
        put(piv, k, p0);
        put(lu, D.x + 1, u01);
        put(lu, D.x + 2 + D.z, l10);
        put(piv, k + 1, pkPivot<T>(b, s, e[3], e[3] - acc[3] - l10 * u01, true));
        return;
    }
    if (kind == kPUpper) {
        const T v0 = e[0] - acc[0];
        put(lu, D.x, v0);
        put(lu, D.y, e[1] - acc[1] - e[2] * v0);
        return;
    }
    const T v0 = (e[0] - acc[0]) / e[3];  // kPLower
    put(lu, D.x, v0);
    put(lu, D.y, (e[1] - acc[1] - v0 * e[2]) / e[4]);
}

__device__ __forceinline__ void clusterArrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void clusterWait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
__device__ __forceinline__ int clusterRank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return (int)r;
}

// Levels [l0, l1) of a schedule (top down for the backward substitution) for the listed system of this cluster; PK:
// the paired schedule (its tasks' second descriptors loaded beside the first). Dynamic shared memory: the walk's
// phases as {first piece, wide, mid-length, end} (16 bytes each).
template <typename T, int W, int C, bool PK>
__global__ void __launch_bounds__(kClusterThreads) k_tail_cluster(DevGrid g, DevBatch b, T* vec, int l0, int l1) {
    constexpr int kClusterWarps = C * kClusterThreads / 32;
    // pairs in flight per lane: the paired schedule's products take up to four operands a pair, so it keeps four (its
    // pieces of more than four pairs go to 8-lane groups)
    constexpr int UF = PK ? 4 : kClusterInFlight;
    extern __shared__ int4 clPhase[];
    const int s = b.activeList[blockIdx.x / C];
    // uniform over the cluster: every CTA of it returns, or none does (no CTA may miss a cluster barrier)
    if (W != kWorkFactor && vec != (T*)b.y && !b.refine[s]) return;
    const int* ptr = PK ? (W == kWorkFactor ? g.pfWorkPtr : (W == kWorkBackward ? g.pbWorkPtr : g.pvWorkPtr))
                        : (W == kWorkFactor ? g.fWorkPtr : (W == kWorkBackward ? g.bWorkPtr : g.vWorkPtr));
    const int4* desc = PK ? (W == kWorkFactor ? g.pfA : (W == kWorkBackward ? g.pbA : g.pvA))
                          : (W == kWorkFactor ? g.fDesc : (W == kWorkBackward ? g.bDesc : g.vDesc));
    const int4* descB = W == kWorkFactor ? g.pfB : (W == kWorkBackward ? g.pbB : g.pvB);
    const int* midCnt = PK ? (W == kWorkFactor ? g.pfMid : (W == kWorkBackward ? g.pbMid : g.pvMid))
                           : (W == kWorkFactor ? g.fMid : (W == kWorkBackward ? g.bMid : g.vMid));
    const int* wide = PK ? (W == kWorkFactor ? g.pfWide : (W == kWorkBackward ? g.pbWide : g.pvWide))
                         : (W == kWorkFactor ? g.fWide : (W == kWorkBackward ? g.bWide : g.vWide));
    const int phases = W == kWorkFactor ? 2 : 1;
    const int nPh = phases * (l1 - l0);
    for (int k = threadIdx.x; k < nPh; k += blockDim.x) {
        const int step = k / phases, ph = k % phases;
        const int l = W == kWorkBackward ? l1 - 1 - step : l0 + step;
        const int i = phases * l + ph;
        clPhase[k] = make_int4(__ldg(ptr + i), __ldg(wide + i), __ldg(midCnt + i), __ldg(ptr + i + 1));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int gw = clusterRank() * (kClusterThreads / 32) + (int)(threadIdx.x >> 5);  // warp of the cluster
    const unsigned gmask = 0xFFu << (lane & 24);
    auto loadPairs = [&](int cls, const int4 d, int2 (&a)[UF]) {
        if (PK) clPairsPOf<W, UF>(g, cls, d, a);
        else clPairsOf<W, UF>(g, cls, d, a);
    };
    // the first unit of this warp two phases deep: its descriptors for phase k + 1, its descriptors and pairs for k
    int clsCur = -1, posCur = -1, clsNext = -1, posNext = -1;
    int4 dCur = make_int4(0, 0, 0, 0), dNext = make_int4(0, 0, 0, 0);
    int4 eCur = make_int4(0, 0, 0, 0), eNext = make_int4(0, 0, 0, 0);
    int2 aCur[UF];
    auto firstOf = [&](int k, int& cls, int& pos, int4& d, int4& e) {
        cls = -1;
        pos = -1;
        if (k < nPh && gw < unitCount(clPhase[k])) {
            pos = unitPiece(clPhase[k], gw, lane, cls);
            if (pos >= 0) {
                d = __ldg(desc + pos);
                if (PK) e = __ldg(descB + pos);
            }
        }
    };
    firstOf(0, clsCur, posCur, dCur, eCur);
    if (posCur >= 0) loadPairs(clsCur, dCur, aCur);
    firstOf(1, clsNext, posNext, dNext, eNext);
    for (int k = 0; k < nPh; k++) {
        const int4 P = clPhase[k];
        const int nu = unitCount(P);
        for (int u = gw; u < nu; u += kClusterWarps) {
            int cls, pos;
            int4 d, e = make_int4(0, 0, 0, 0);
            int2 a[UF];
            if (u == gw) {
                cls = clsCur;
                pos = posCur;
                d = dCur;
                e = eCur;
#pragma unroll
                for (int q = 0; q < UF; q++) a[q] = aCur[q];
            } else {
                pos = unitPiece(P, u, lane, cls);
                if (pos >= 0) {
                    d = __ldg(desc + pos);
                    if (PK) e = __ldg(descB + pos);
                    loadPairs(cls, d, a);
                }
            }
            if (PK) {
                if (cls == 0) clRunP<T, W, 32, UF>(g, b, vec, d, e, a, s, 0xffffffffu);          // pos warp-uniform
                else if (cls == 1) { if (pos >= 0) clRunP<T, W, 8, UF>(g, b, vec, d, e, a, s, gmask); }  // group-uniform
                else if (pos >= 0) clRunP<T, W, 1, UF>(g, b, vec, d, e, a, s, 0u);
            } else {
                if (cls == 0) clRun<T, W, 32, UF>(g, b, vec, d, a, s, 0xffffffffu);
                else if (cls == 1) { if (pos >= 0) clRun<T, W, 8, UF>(g, b, vec, d, a, s, gmask); }
                else if (pos >= 0) clRun<T, W, 1, UF>(g, b, vec, d, a, s, 0u);
            }
        }
        __syncwarp();  // the barrier below is .aligned: every warp arrives converged
        clusterArrive();
        // static data only, safe before the acquire: the next phase's first pairs, the phase after's descriptors
        clsCur = clsNext;
        posCur = posNext;
        dCur = dNext;
        eCur = eNext;
        if (posCur >= 0) loadPairs(clsCur, dCur, aCur);
        firstOf(k + 2, clsNext, posNext, dNext, eNext);
        clusterWait();
    }
}

inline size_t ClusterSmemBytes(int nLevels) { return (size_t)2 * nLevels * sizeof(int4); }

// Launch a walk of levels [l0, l1) for the nActive listed systems of b, one cluster of C CTAs per system.
template <typename T, int W, int C, bool PK>
cudaError_t LaunchTailClusterC(const DevGrid& g, const DevBatch& b, T* vec, int l0, int l1, int nActive, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nActive * C);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = ClusterSmemBytes(l1 - l0);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_tail_cluster<T, W, C, PK>, g, b, vec, l0, l1);
}
template <typename T, int W, bool PK>
cudaError_t LaunchTailClusterK(const DevGrid& g, const DevBatch& b, T* vec, int l0, int l1, int nActive, cudaStream_t st) {
    switch (ClusterCtasFor(nActive)) {
        case 16: return LaunchTailClusterC<T, W, 16, PK>(g, b, vec, l0, l1, nActive, st);
        case 8: return LaunchTailClusterC<T, W, 8, PK>(g, b, vec, l0, l1, nActive, st);
        case 4: return LaunchTailClusterC<T, W, 4, PK>(g, b, vec, l0, l1, nActive, st);
        case 2: return LaunchTailClusterC<T, W, 2, PK>(g, b, vec, l0, l1, nActive, st);
        default: return LaunchTailClusterC<T, W, 1, PK>(g, b, vec, l0, l1, nActive, st);
    }
}
// Levels [l0, l1) of the paired schedule (paired) or of the scalar one.
template <typename T, int W>
cudaError_t LaunchTailCluster(const DevGrid& g, const DevBatch& b, T* vec, int l0, int l1, int nActive, cudaStream_t st,
                              bool paired) {
    return paired ? LaunchTailClusterK<T, W, true>(g, b, vec, l0, l1, nActive, st)
                  : LaunchTailClusterK<T, W, false>(g, b, vec, l0, l1, nActive, st);
}

}  // namespace gs
