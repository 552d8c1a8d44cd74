// gs_cluster.cuh — the few-systems path on thread-block clusters (sm_100a).
//
// When only a handful of systems are still stepping (the outages that never converge run to the iteration cap, as in
// the reference), one CTA per system leaves most of the GPU idle and walks ~400 level phases with the latency of one
// SM's loads. Here every listed system gets a cluster of kClusterCtas CTAs on as many SMs: each level (and phase) of
// a schedule is dealt out over all warps of the cluster, and a cluster barrier (barrier.cluster.arrive.release /
// wait.acquire) separates the levels. The walk covers every level, so the per-level launches of the wide bottom
// levels go away too.
//
// Coherence: the CTAs of a cluster run on different SMs, whose L1 caches do not see each other's stores, so every
// value another CTA may have written during the walk (LU entries, pivots, right-hand sides) is read with
// ld.global.cg (L2) and written with st.global.cg. The barrier's release / acquire at cluster scope orders those
// stores before the loads of the next level. Index data (descriptors, pairs, rows) never changes and is read through
// the read-only path.
//
// The work of a level is dealt statically: wide pieces to warps, mid-length pieces to 8-lane groups, short pieces to
// threads, round-robin over the cluster. Each piece is summed in the same lane order as the one-CTA walk (k_tail), so
// a system's arithmetic does not depend on which walk ran it.
#pragma once
#include <cooperative_groups.h>

namespace gs {

constexpr int kClusterCtas = 8;        // CTAs per system (the portable cluster size)
constexpr int kClusterThreads = 1024;  // threads per CTA
constexpr int kClusterWarps = kClusterCtas * kClusterThreads / 32;
constexpr int kClusterMaxSystems = 16; // more systems than this: one CTA each (k_tail) keeps the GPU fuller

template <typename T>
__device__ __forceinline__ T ldL2(const T* p) { return __ldcg(p); }
template <typename T>
__device__ __forceinline__ void stL2(T* p, T v) { __stcg(p, v); }

// sum over pairs [q0, q1) of lu[a] * rhs[c] for system s by a group of G lanes (G = 32, 8 or 1): lane j takes pairs
// q0 + j, q0 + j + G, ..., four in flight, then a fixed butterfly over the group (mask: its lanes)
template <typename T, int G>
__device__ __forceinline__ T clDot(const T* lu, const T* rhs, const int2* __restrict__ pr, int64_t q0, int64_t q1,
                                   size_t B, int s, unsigned mask) {
    const int j = G == 1 ? 0 : (int)(threadIdx.x & (G - 1));
    T acc = T(0);
    for (int64_t q = q0 + j; q < q1; q += 4 * G) {
        int2 a[4];
#pragma unroll
        for (int u = 0; u < 4; u++) a[u] = q + u * G < q1 ? __ldg(pr + q + u * G) : make_int2(-1, -1);
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
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(mask, acc, off);
    return acc;
}

// sum over the U row of backward node d (x(r) for r in P_k) by a group of G lanes
template <typename T, int G>
__device__ __forceinline__ T clBackDot(const T* lu, const T* y, const int* __restrict__ pRows, const int4 d, size_t B,
                                       int s, unsigned mask) {
    const int j = G == 1 ? 0 : (int)(threadIdx.x & (G - 1));
    const int64_t base = d.y;
    const int c = d.z;
    const int* rows = pRows + d.w;
    T acc = T(0);
    for (int t = j; t < c; t += 4 * G) {
        int r[4];
#pragma unroll
        for (int u = 0; u < 4; u++) r[u] = t + u * G < c ? __ldg(rows + t + u * G) : -1;
        T uu[4], x[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const bool ok = r[u] >= 0;
            uu[u] = ok ? ldL2(lu + (size_t)(base + 1 + t + u * G) * B + s) : T(0);
            x[u] = ok ? ldL2(y + (size_t)r[u] * B + s) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) acc += uu[u] * x[u];
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(mask, acc, off);
    return acc;
}

// One piece of a schedule by a group of G lanes; the group's first lane writes the result.
template <typename T, int W, int G>
__device__ __forceinline__ void clPiece(const DevGrid& g, const DevBatch& b, T* vec, const int4 d, int s, unsigned mask) {
    const size_t B = (size_t)b.B;
    T* lu = (T*)b.lu;
    const bool lead = G == 1 || (threadIdx.x & (G - 1)) == 0;
    if (W == kWorkBackward) {
        const T acc = clBackDot<T, G>(lu, vec, g.pRows, d, B, s, mask);
        if (lead) {
            const int k = d.x;
            stL2(vec + (size_t)k * B + s, (ldL2(vec + (size_t)k * B + s) - acc) / ldL2((const T*)b.piv + (size_t)k * B + s));
        }
        return;
    }
    if (W == kWorkForward) {
        const T dot = clDot<T, G>(lu, vec, g.pairs, d.y, d.z, B, s, mask);
        if (lead) {
            T* p = vec + (size_t)descNode(d) * B + s;
            stL2(p, ldL2(p) - dot);
        }
        return;
    }
    const int kind = descKind(d), slot = d.x, node = descNode(d);
    T* y = (T*)b.y;
    const T dot = clDot<T, G>(lu, kind == kFwd ? y : lu, g.pairs, d.y, d.z, B, s, mask);
    if (!lead) return;
    if (kind == kFwd) {
        T* p = y + (size_t)slot * B + s;
        stL2(p, ldL2(p) - dot);
        return;
    }
    const T a = descHasA(d) ? ldL2(lu + (size_t)slot * B + s) : T(0);
    T v = a - dot;
    if (kind == kDiag) {
        const T fl = pivotFloor<T>() * (fabs(a) > T(1) ? fabs(a) : T(1));
        if (!(fabs(v) > fl)) { atomicOr(&b.flags[s], kFlagPivotPerturbed); v = (v < T(0)) ? -fl : fl; }
        stL2((T*)b.piv + (size_t)node * B + s, v);
        return;
    }
    if (kind == kLower) v = v / ldL2((const T*)b.piv + (size_t)node * B + s);
    stL2(lu + (size_t)slot * B + s, v);
}

// Levels [l0, l1) of a schedule (top down for the backward substitution) for the listed system of this cluster.
template <typename T, int W>
__global__ void __launch_bounds__(kClusterThreads) k_tail_cluster(DevGrid g, DevBatch b, T* vec, int l0, int l1) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int s = b.activeList[blockIdx.x / kClusterCtas];
    // uniform over the cluster: every CTA of it returns, or none does (no CTA may miss a cluster barrier)
    if (W != kWorkFactor && vec != (T*)b.y && !b.refine[s]) return;
    const int* ptr = W == kWorkFactor ? g.fWorkPtr : (W == kWorkBackward ? g.bWorkPtr : g.vWorkPtr);
    const int4* desc = W == kWorkFactor ? g.fDesc : (W == kWorkBackward ? g.bDesc : g.vDesc);
    const int* midCnt = W == kWorkFactor ? g.fMid : (W == kWorkBackward ? g.bMid : g.vMid);
    const int* wide = W == kWorkFactor ? g.fWide : (W == kWorkBackward ? g.bWide : g.vWide);
    constexpr int G = 8;
    const int lane = threadIdx.x & 31;
    const int gw = (int)cl.block_rank() * (kClusterThreads / 32) + (int)(threadIdx.x >> 5);  // warp of the cluster
    const unsigned gmask = 0xFFu << (lane & 24);
    const int phases = W == kWorkFactor ? 2 : 1;
    for (int step = 0; step < l1 - l0; step++) {
        const int l = W == kWorkBackward ? l1 - 1 - step : l0 + step;
        for (int ph = 0; ph < phases; ph++) {
            const int i = phases * l + ph;
            const int w0 = __ldg(ptr + i), w1 = __ldg(ptr + i + 1), nw = __ldg(wide + i), nm = __ldg(midCnt + i);
            for (int p = gw; p < nw; p += kClusterWarps) clPiece<T, W, 32>(g, b, vec, __ldg(desc + w0 + p), s, 0xffffffffu);
            for (int p = gw * 4 + (lane >> 3); p < nm; p += kClusterWarps * 4)
                clPiece<T, W, G>(g, b, vec, __ldg(desc + w0 + nw + p), s, gmask);
            const int nr = w1 - w0 - nw - nm;
            for (int p = gw * 32 + lane; p < nr; p += kClusterWarps * 32)
                clPiece<T, W, 1>(g, b, vec, __ldg(desc + w0 + nw + nm + p), s, 0u);
            cl.sync();
        }
    }
}

// Launch a cluster walk of levels [l0, l1) for the nActive listed systems of b.
template <typename T, int W>
cudaError_t LaunchTailCluster(const DevGrid& g, const DevBatch& b, T* vec, int l0, int l1, int nActive, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nActive * kClusterCtas);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = 0;
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
