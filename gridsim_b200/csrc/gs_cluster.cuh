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

constexpr int kClusterCtas = 8;        // CTAs per system (the portable cluster size)
constexpr int kClusterThreads = 512;   // threads per CTA
constexpr int kClusterWarps = kClusterCtas * kClusterThreads / 32;
constexpr int kClusterMaxSystems = 16; // more systems than this: one CTA each (k_tail) keeps the GPU fuller
constexpr size_t kClusterSmemMax = 64 * 1024;  // the per-phase table in shared memory (16 bytes a phase)

template <typename T>
__device__ __forceinline__ T ldL2(const T* p) { return __ldcg(p); }
template <typename T>
__device__ __forceinline__ void stL2(T* p, T v) { __stcg(p, v); }

// A piece and its first round of index pairs for this lane, loaded ahead: (LU slot, right-hand-side index) for
// factorisation and forward entries, (U slot, row) for a backward node; x = -1 past the end.
struct Ahead {
    int4 d;
    int2 a[4];
};

template <int W, int G>
__device__ __forceinline__ void clLoadAhead(const DevGrid& g, const int4* __restrict__ desc, int pos, Ahead& x) {
    x.d = __ldg(desc + pos);
    const int j = G == 1 ? 0 : (int)(threadIdx.x & (G - 1));
    if (W == kWorkBackward) {
        const int c = x.d.z;
        const int base = x.d.y;  // LU slots fit 32 bits (checked by the symbolic analysis)
        const int* rows = g.pRows + x.d.w;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int t = j + u * G;
            x.a[u] = t < c ? make_int2(base + 1 + t, __ldg(rows + t)) : make_int2(-1, -1);
        }
    } else {
        const int q0 = x.d.y, q1 = x.d.z;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int q = q0 + j + u * G;
            x.a[u] = q < q1 ? __ldg(g.pairs + q) : make_int2(-1, -1);
        }
    }
}

// One piece by a group of G lanes (G = 32, 8 or 1) from its loaded-ahead first round; the group's first lane writes.
// Lane j of the group takes pairs j, j + G, ..., four in flight per round, then a fixed butterfly over the group.
template <typename T, int W, int G>
__device__ __forceinline__ void clRun(const DevGrid& g, const DevBatch& b, T* vec, const Ahead& x, int s, unsigned mask) {
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    T* piv = (T*)b.piv;
    const int4 d = x.d;
    const int j = G == 1 ? 0 : (int)(threadIdx.x & (G - 1));
    const bool lead = j == 0;
    // where the result goes and what it combines with, loaded beside the first operands
    T* out;
    const T* rhs;
    T base = T(0), div = T(1);
    int kind = kUpper;
    bool hasA = true;
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
        hasA = descHasA(d);
        const int node = descNode(d);
        T* y = (T*)b.y;
        rhs = kind == kFwd ? y : lu;
        out = kind == kFwd ? y + (size_t)d.x * B + s
                           : (kind == kDiag ? piv + (size_t)node * B + s : lu + (size_t)d.x * B + s);
        if (lead) {
            if (kind == kFwd) base = ldL2(out);
            else if (hasA) base = ldL2(lu + (size_t)d.x * B + s);
            if (kind == kLower) div = ldL2(piv + (size_t)node * B + s);
        }
    }
    T acc = T(0);
    {
        T l[4], r[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const bool ok = x.a[u].x >= 0;
            l[u] = ok ? ldL2(lu + (size_t)x.a[u].x * B + s) : T(0);
            r[u] = ok ? ldL2(rhs + (size_t)x.a[u].y * B + s) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) acc += l[u] * r[u];
    }
    // further rounds (pieces longer than 4 G)
    if (W == kWorkBackward) {
        const int c = d.z;
        const int* rows = g.pRows + d.w;
        for (int t = j + 4 * G; t < c; t += 4 * G) {
            int rr[4];
#pragma unroll
            for (int u = 0; u < 4; u++) rr[u] = t + u * G < c ? __ldg(rows + t + u * G) : -1;
            T uu[4], xv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const bool ok = rr[u] >= 0;
                uu[u] = ok ? ldL2(lu + (size_t)(d.y + 1 + t + u * G) * B + s) : T(0);
                xv[u] = ok ? ldL2(vec + (size_t)rr[u] * B + s) : T(0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) acc += uu[u] * xv[u];
        }
    } else {
        const int q1 = d.z;
        for (int q = d.y + j + 4 * G; q < q1; q += 4 * G) {
            int2 a[4];
#pragma unroll
            for (int u = 0; u < 4; u++) a[u] = q + u * G < q1 ? __ldg(g.pairs + q + u * G) : make_int2(-1, -1);
            T l[4], r[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const bool ok = a[u].x >= 0;
                l[u] = ok ? ldL2(lu + (size_t)a[u].x * B + s) : T(0);
                r[u] = ok ? ldL2(rhs + (size_t)a[u].y * B + s) : T(0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) acc += l[u] * r[u];
        }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(mask, acc, off);
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
template <typename T, int W>
__global__ void __launch_bounds__(kClusterThreads) k_tail_cluster(DevGrid g, DevBatch b, T* vec, int l0, int l1) {
    extern __shared__ int4 clPhase[];
    const int s = b.activeList[blockIdx.x / kClusterCtas];
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
    const int pm0 = gw * 4 + (lane >> 3);  // this 8-lane group's first mid-length piece
    const int ps0 = gw * 32 + lane;        // this thread's first short piece
    const unsigned gmask = 0xFFu << (lane & 24);
    Ahead aw, am, as;
    auto ahead = [&](int k) {
        const int4 P = clPhase[k];  // {w0, nw, nm, w1}
        if (gw < P.y) clLoadAhead<W, 32>(g, desc, P.x + gw, aw);
        if (pm0 < P.z) clLoadAhead<W, 8>(g, desc, P.x + P.y + pm0, am);
        if (ps0 < P.w - P.x - P.y - P.z) clLoadAhead<W, 1>(g, desc, P.x + P.y + P.z + ps0, as);
    };
    if (nPh > 0) ahead(0);
    for (int k = 0; k < nPh; k++) {
        const int4 P = clPhase[k];
        const int w0 = P.x, nw = P.y, nm = P.z, nr = P.w - P.x - P.y - P.z;
        for (int p = gw; p < nw; p += kClusterWarps) {
            if (p != gw) clLoadAhead<W, 32>(g, desc, w0 + p, aw);
            clRun<T, W, 32>(g, b, vec, aw, s, 0xffffffffu);
        }
        for (int p = pm0; p < nm; p += kClusterWarps * 4) {
            if (p != pm0) clLoadAhead<W, 8>(g, desc, w0 + nw + p, am);
            clRun<T, W, 8>(g, b, vec, am, s, gmask);
        }
        for (int p = ps0; p < nr; p += kClusterWarps * 32) {
            if (p != ps0) clLoadAhead<W, 1>(g, desc, w0 + nw + nm + p, as);
            clRun<T, W, 1>(g, b, vec, as, s, 0u);
        }
        __syncwarp();  // the barrier below is .aligned: every warp arrives converged
        clusterArrive();
        if (k + 1 < nPh) ahead(k + 1);  // static data only: safe before the acquire
        clusterWait();
    }
}

inline size_t ClusterSmemBytes(int nLevels) { return (size_t)2 * nLevels * sizeof(int4); }

// Launch a cluster walk of levels [l0, l1) for the nActive listed systems of b.
template <typename T, int W>
cudaError_t LaunchTailCluster(const DevGrid& g, const DevBatch& b, T* vec, int l0, int l1, int nActive, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nActive * kClusterCtas);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = ClusterSmemBytes(l1 - l0);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClusterCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_tail_cluster<T, W>, g, b, vec, l0, l1);
}

}  // namespace gs
