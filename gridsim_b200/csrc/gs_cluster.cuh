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

constexpr int kClusterCtas = 8;        // the largest cluster: CTAs per system (the portable cluster size)
constexpr int kClusterThreads = 512;   // threads per CTA (one CTA per SM at the walk's register count)
constexpr int kClusterMaxSystems = 296; // more systems than this: the full-batch step
// CTAs per system for n systems: as many as keep the systems' clusters within about one wave of the 148 SMs
inline int ClusterCtasFor(int n) { return n <= 18 ? 8 : n <= 37 ? 4 : n <= 74 ? 2 : 1; }
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
template <int W, int G>
__device__ __forceinline__ void clPairs(const DevGrid& g, const int4 d, int2 (&a)[kClusterInFlight]) {
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
template <int W>
__device__ __forceinline__ void clPairsOf(const DevGrid& g, int cls, const int4 d, int2 (&a)[kClusterInFlight]) {
    if (cls == 0) clPairs<W, 32>(g, d, a);
    else if (cls == 1) clPairs<W, 8>(g, d, a);
    else clPairs<W, 1>(g, d, a);
}

// One piece by a group of G lanes (G = 32, 8 or 1) from its loaded first round; the group's first lane writes. Lane j
// of the group takes pairs j, j + G, ..., kClusterInFlight in flight per round, then a fixed butterfly over the group.
template <typename T, int W, int G>
__device__ __forceinline__ void clRun(const DevGrid& g, const DevBatch& b, T* vec, const int4 d,
                                      const int2 (&a0)[kClusterInFlight], int s, unsigned mask) {
    constexpr int U = kClusterInFlight;
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

__device__ __forceinline__ void clusterArrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void clusterWait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
__device__ __forceinline__ int clusterRank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return (int)r;
}

// Levels [l0, l1) of a schedule (top down for the backward substitution) for the listed system of this cluster.
// Dynamic shared memory: the walk's phases as {first piece, wide, mid-length, end} (16 bytes each).
template <typename T, int W, int C>
__global__ void __launch_bounds__(kClusterThreads) k_tail_cluster(DevGrid g, DevBatch b, T* vec, int l0, int l1) {
    constexpr int kClusterWarps = C * kClusterThreads / 32;
    extern __shared__ int4 clPhase[];
    const int s = b.activeList[blockIdx.x / C];
    // uniform over the cluster: every CTA of it returns, or none does (no CTA may miss a cluster barrier)
    if (W != kWorkFactor && vec != (T*)b.y && !b.refine[s]) return;
    const int* ptr = W == kWorkFactor ? g.fWorkPtr : (W == kWorkBackward ? g.bWorkPtr : g.vWorkPtr);
    const int4* desc = W == kWorkFactor ? g.fDesc : (W == kWorkBackward ? g.bDesc : g.vDesc);
    const int* midCnt = W == kWorkFactor ? g.fMid : (W == kWorkBackward ? g.bMid : g.vMid);
    const int* wide = W == kWorkFactor ? g.fWide : (W == kWorkBackward ? g.bWide : g.vWide);
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
    // the first unit of this warp two phases deep: its descriptor for phase k + 1, its descriptor and pairs for k
    int clsCur = -1, posCur = -1, clsNext = -1, posNext = -1;
    int4 dCur = make_int4(0, 0, 0, 0), dNext = make_int4(0, 0, 0, 0);
    int2 aCur[kClusterInFlight];
    auto firstOf = [&](int k, int& cls, int& pos, int4& d) {
        cls = -1;
        pos = -1;
        if (k < nPh && gw < unitCount(clPhase[k])) {
            pos = unitPiece(clPhase[k], gw, lane, cls);
            if (pos >= 0) d = __ldg(desc + pos);
        }
    };
    firstOf(0, clsCur, posCur, dCur);
    if (posCur >= 0) clPairsOf<W>(g, clsCur, dCur, aCur);
    firstOf(1, clsNext, posNext, dNext);
    for (int k = 0; k < nPh; k++) {
        const int4 P = clPhase[k];
        const int nu = unitCount(P);
        for (int u = gw; u < nu; u += kClusterWarps) {
            int cls, pos;
            int4 d;
            int2 a[kClusterInFlight];
            if (u == gw) {
                cls = clsCur;
                pos = posCur;
                d = dCur;
#pragma unroll
                for (int q = 0; q < kClusterInFlight; q++) a[q] = aCur[q];
            } else {
                pos = unitPiece(P, u, lane, cls);
                if (pos >= 0) {
                    d = __ldg(desc + pos);
                    clPairsOf<W>(g, cls, d, a);
                }
            }
            if (cls == 0) clRun<T, W, 32>(g, b, vec, d, a, s, 0xffffffffu);          // pos is warp-uniform here
            else if (cls == 1) { if (pos >= 0) clRun<T, W, 8>(g, b, vec, d, a, s, gmask); }  // group-uniform
            else if (pos >= 0) clRun<T, W, 1>(g, b, vec, d, a, s, 0u);
        }
        __syncwarp();  // the barrier below is .aligned: every warp arrives converged
        clusterArrive();
        // static data only, safe before the acquire: the next phase's first pairs, the phase after's descriptor
        clsCur = clsNext;
        posCur = posNext;
        dCur = dNext;
        if (posCur >= 0) clPairsOf<W>(g, clsCur, dCur, aCur);
        firstOf(k + 2, clsNext, posNext, dNext);
        clusterWait();
    }
}

inline size_t ClusterSmemBytes(int nLevels) { return (size_t)2 * nLevels * sizeof(int4); }

// Launch a walk of levels [l0, l1) for the nActive listed systems of b, one cluster of C CTAs per system.
template <typename T, int W, int C>
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
    return cudaLaunchKernelEx(&cfg, k_tail_cluster<T, W, C>, g, b, vec, l0, l1);
}
template <typename T, int W>
cudaError_t LaunchTailCluster(const DevGrid& g, const DevBatch& b, T* vec, int l0, int l1, int nActive, cudaStream_t st) {
    switch (ClusterCtasFor(nActive)) {
        case 8: return LaunchTailClusterC<T, W, 8>(g, b, vec, l0, l1, nActive, st);
        case 4: return LaunchTailClusterC<T, W, 4>(g, b, vec, l0, l1, nActive, st);
        case 2: return LaunchTailClusterC<T, W, 2>(g, b, vec, l0, l1, nActive, st);
        default: return LaunchTailClusterC<T, W, 1>(g, b, vec, l0, l1, nActive, st);
    }
}

}  // namespace gs
