// gs_multi.cuh — the uneven multi-grid batch (gs_pf_solve_multi of include/gridsim_b200.h). Part of gs_engine.cu's
// translation unit: it runs the engine's per-bus and per-level device functions inside one persistent kernel.
//
// k_newton: a persistent CTA takes the next (grid, case) item from a device counter (items sorted largest grid
// first, so that the long solves start early and the short ones fill in behind them) and runs that case's whole
// Newton iteration with block barriers only: mismatch + Jacobian over its buses, the status test, the level walk of
// the factorisation and the triangular solves (walkLevels, as the few-systems path), the FP64 refinement in mixed
// precision, max |dx| and the damped update. A case's state lives in the CTA's slot of an arena sized for the
// largest grid, system-major (interleave stride 1). The launch is captured in a CUDA graph with the reset of the
// item counter. The CTA size, and whether the top of each grid's elimination tree is walked in shared memory (which
// takes L1 capacity from the levels below it), are the autotuner's: each candidate runs on a sample of the items and
// the fastest is kept for the set of grids.
#pragma once

#include <map>

namespace gs {

struct MultiItem {
    int grid;
    int caseIdx;   // index of the case in the per-case outputs
    int64_t off;   // offset of the case's buses in the concatenated per-bus arrays
};

// Newton control words of one slot
struct SlotScalars {
    unsigned long long maxMis, maxDx;
    double startMis, finalMis;
    int status, iters, convIters, active, flags, outage, refine, activeCount[2], activeList[1];
};

struct SlotArena {
    char* base;
    size_t stride;  // bytes per slot
    size_t offLu, offPiv, offY, offZ, offRhs, offVm, offVa, offScal;
};

__device__ __forceinline__ double blockMaxD(double v, double* red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    double r = red[0];
    for (int k = 1; k < nw; k++) r = fmax(r, red[k]);
    return r;
}

__device__ __forceinline__ int blockOrI(int v, int* red) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, off);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    int r = 0;
    for (int k = 0; k < nw; k++) r |= red[k];
    return r;
}

template <typename T>
__global__ void __launch_bounds__(1024) k_newton(const DevGrid* grids, const MultiItem* items, int nItems, int* next,
                                                 SlotArena arena, const double* loadScale, const int* outage,
                                                 int* outStatus, int* outIters, double* outMis, double* outVm,
                                                 double* outVa, double tol, double divLimit, int maxIter,
                                                 unsigned long long* steps, int useTopFlag, int queueOffset) {
    __shared__ DevGrid sg;
    __shared__ int sItem, sGo;
    __shared__ double redD[32];
    __shared__ int redI[32];
    const int tid = threadIdx.x, bd = blockDim.x;
    char* base = arena.base + (size_t)blockIdx.x * arena.stride;
    SlotScalars* sc = reinterpret_cast<SlotScalars*>(base + arena.offScal);
    const bool mixed = sizeof(T) < sizeof(double);
    T* sm = reinterpret_cast<T*>(gsTopSmem);  // the top part of the current item's grid
    const bool useTop = useTopFlag != 0;
    int* queue = reinterpret_cast<int*>(gsTopSmem + queueOffset);  // the level walks' piece counters
    for (;;) {
        if (tid == 0) sItem = atomicAdd(next, 1);
        __syncthreads();
        const int it = sItem;
        if (it >= nItems) return;
        const MultiItem item = items[it];
        {
            const int* src = reinterpret_cast<const int*>(grids + item.grid);
            int* dst = reinterpret_cast<int*>(&sg);
            for (int k = tid; k < (int)(sizeof(DevGrid) / sizeof(int)); k += bd) dst[k] = src[k];
        }
        __syncthreads();
        const DevGrid& g = sg;
        const int n = g.n, m = g.m;
        DevBatch b{};
        b.B = 1;
        b.count = 1;
        b.nLevels = g.nLevels;
        b.vm = reinterpret_cast<double*>(base + arena.offVm);
        b.va = reinterpret_cast<double*>(base + arena.offVa);
        b.lu = base + arena.offLu;
        b.piv = base + arena.offPiv;
        b.y = base + arena.offY;
        b.z = mixed ? base + arena.offZ : nullptr;
        b.rhs64 = mixed ? reinterpret_cast<double*>(base + arena.offRhs) : nullptr;
        b.refine = mixed ? &sc->refine : nullptr;
        b.maxMis = &sc->maxMis;
        b.maxDx = &sc->maxDx;
        b.startMis = &sc->startMis;
        b.finalMis = &sc->finalMis;
        b.status = &sc->status;
        b.iters = &sc->iters;
        b.convIters = &sc->convIters;
        b.active = &sc->active;
        b.flags = &sc->flags;
        b.outage = &sc->outage;
        b.loadScale = loadScale ? loadScale + item.off : nullptr;
        b.activeCount = sc->activeCount;
        b.activeList = sc->activeList;
        // the case's stored voltages (PV and slack magnitudes and the slack angle are the set points already)
        for (int i = tid; i < n; i += bd) {
            b.vm[i] = g.vm0[i];
            b.va[i] = g.va0[i];
        }
        if (tid == 0) {
            sc->maxMis = 0ull;
            sc->maxDx = 0ull;
            sc->startMis = 0.0;
            sc->finalMis = NAN;
            sc->status = GS_PF_MAX_ITERATIONS;
            sc->iters = 0;
            sc->convIters = 0;
            sc->active = 1;
            sc->flags = 0;
            sc->outage = outage ? outage[item.caseIdx] : -1;
            sc->refine = 0;
        }
        __syncthreads();
        for (int iter = 0;; iter++) {
            double lm = 0.0;
            int bad = 0;
            for (int i = tid; i < n; i += bd) busMismatchJac<T>(g, b, i, 0, 1, nullptr, nullptr, lm, bad);
            lm = blockMaxD(lm, redD);
            bad = blockOrI(bad, redI);
            if (tid == 0) {
                if (lm > 0.0) sc->maxMis = (unsigned long long)__double_as_longlong(lm);
                if (bad & 1) sc->flags |= kFlagNonFinite;
                if (bad & 2) sc->flags |= kFlagJacBad;
                sc->activeCount[0] = sc->activeCount[1] = 0;
                sGo = statusStep(b, 0, iter, tol, divLimit, maxIter) ? 1 : 0;
            }
            __syncthreads();
            if (!sGo) break;
            factorSystem<T>(g, b, 0, sm, useTop, queue);
            backwardSystem<T>(g, b, (T*)b.y, 0, sm, useTop, queue);
            const int refine = mixed ? sc->refine : 0;
            if (refine) {
                for (int i = tid; i < n; i += bd) busResidual<T>(g, b, i, 0);
                __syncthreads();
                forwardSystem<T>(g, b, (T*)b.z, 0, sm, useTop, queue);
                backwardSystem<T>(g, b, (T*)b.z, 0, sm, useTop, queue);
            }
            const T* y = (const T*)b.y;
            const T* z = (const T*)b.z;
            double mx = 0.0;
            int badStep = 0;
            for (int k = tid; k < m; k += bd) {
                const double v = (double)y[k] + (refine ? (double)z[k] : 0.0);
                badStep |= isfinite(v) ? 0 : 1;
                mx = fmax(mx, fabs(v));
            }
            mx = blockMaxD(mx, redD);
            badStep = blockOrI(badStep, redI);
            if (tid == 0) {
                sc->maxDx = (unsigned long long)__double_as_longlong(mx);
                if (badStep) sc->flags |= kFlagStepBad;
            }
            __syncthreads();
            if (!badStep)
                for (int i = tid; i < n; i += bd) busUpdate<T>(g, b, i, 0, refine);
            __syncthreads();
        }
        for (int i = tid; i < n; i += bd) {
            if (outVm) outVm[item.off + i] = b.vm[i];
            if (outVa) outVa[item.off + i] = b.va[i] * (180.0 / 3.14159265358979323846);
        }
        if (tid == 0) {
            outStatus[item.caseIdx] = sc->status;
            outIters[item.caseIdx] = sc->iters;
            outMis[item.caseIdx] = sc->finalMis;
            atomicAdd(steps, (unsigned long long)sc->iters);
        }
        __syncthreads();
    }
}

}  // namespace gs

extern "C" int gs_pf_solve_multi(gs_ctx* ctx, int32_t nGrids, gs_grid* const* grids, const int32_t* counts,
                                 const double* loadScale, const int32_t* outage, const gs_pf_opts* opts,
                                 int32_t* status, int32_t* iterations, double* maxMismatch, double* vmOut,
                                 double* vaOut, gs_multi_stats* stats) {
    using namespace gs;
    if (!ctx || nGrids < 0 || (nGrids > 0 && (!grids || !counts))) return GS_ERR_INVALID_ARG;
    int rc = CheckOpts(ctx, opts);
    if (rc) return rc;
    const gs_pf_opts o = *opts;
    if (o.flat_start) return SetErr(ctx, GS_ERR_UNSUPPORTED, "flat_start: pass a flat start in the descriptor");
    // cases, their offsets and the sizes of the largest grid
    int64_t nCases = 0, nStates = 0;
    int maxN = 1, maxM = 1;
    int64_t maxLu = 1;
    std::vector<int64_t> caseBase(nGrids), stateBase(nGrids);
    for (int k = 0; k < nGrids; k++) {
        if (!grids[k] || counts[k] < 0) return SetErr(ctx, GS_ERR_INVALID_ARG, "grid " + std::to_string(k) + ": null or negative count");
        if (grids[k]->ctx != ctx) return SetErr(ctx, GS_ERR_INVALID_ARG, "grid " + std::to_string(k) + " belongs to another context");
        caseBase[k] = nCases;
        stateBase[k] = nStates;
        nCases += counts[k];
        nStates += (int64_t)counts[k] * grids[k]->sym.n;
        if (counts[k] > 0) {
            maxN = std::max(maxN, grids[k]->sym.n);
            maxM = std::max(maxM, grids[k]->sym.m);
            maxLu = std::max(maxLu, grids[k]->sym.nnzLU);
        }
    }
    if (nCases > (int64_t)INT32_MAX / 2) return SetErr(ctx, GS_ERR_INVALID_ARG, "too many cases");
    if (outage)
        for (int k = 0; k < nGrids; k++)
            for (int c = 0; c < counts[k]; c++) {
                const int ob = outage[caseBase[k] + c];
                const HostGrid& h = grids[k]->host;
                if (ob < -1 || ob >= h.nbr || (ob >= 0 && !h.brOn[ob]))
                    return SetErr(ctx, GS_ERR_INVALID_ARG, "outage " + std::to_string(ob) + " of grid " + std::to_string(k) +
                                                           " is not an in-service branch");
            }
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (nCases == 0) return GS_OK;
    GS_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    // Q limits and the DC retry (ContingencyAnalysis.StudyOptions, ContingencyAnalysis.cs:263-268): a case's system
    // changes between Newton passes, which the one-CTA-per-case solve does not carry; each grid's cases then run as
    // one batch solve (the load scales, outages and states of a grid are contiguous in both layouts). So do cases
    // under partial pivoting, whose steps the batch solve takes with the per-system partial-pivoting factorisation.
    if (o.enforce_q_limits || o.retry_from_dc_start || o.partial_pivoting) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        GS_CUDA(cudaEventCreate(&e0));
        GS_CUDA(cudaEventCreate(&e1));
        struct Events { cudaEvent_t a, b; ~Events() { cudaEventDestroy(a); cudaEventDestroy(b); } } evs{e0, e1};
        GS_CUDA(cudaEventRecord(e0, st));
        for (int k = 0; k < nGrids; k++) {
            if (counts[k] == 0) continue;
            const int64_t c0 = caseBase[k], s0 = stateBase[k];
            rc = gs_pf_solve_batch(grids[k], counts[k], loadScale ? loadScale + s0 : nullptr, outage ? outage + c0 : nullptr,
                                   &o, status ? status + c0 : nullptr, iterations ? iterations + c0 : nullptr,
                                   maxMismatch ? maxMismatch + c0 : nullptr, vmOut ? vmOut + s0 : nullptr,
                                   vaOut ? vaOut + s0 : nullptr);
            if (rc) return rc;
        }
        GS_CUDA(cudaEventRecord(e1, st));
        GS_CUDA(cudaEventSynchronize(e1));
        if (stats) {
            float ms = 0;
            GS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            stats->device_ms = ms;
            stats->items = (int32_t)nCases;
            if (iterations)
                for (int64_t c = 0; c < nCases; c++) stats->system_steps += iterations[c];
        }
        return GS_OK;
    }
    // items, largest grid first (a grid's cases stay together, in case order)
    std::vector<int> order(nGrids);
    for (int k = 0; k < nGrids; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return grids[a]->sym.nnzLU + grids[a]->sym.nnzJ > grids[b]->sym.nnzLU + grids[b]->sym.nnzJ;
    });
    std::vector<MultiItem> items;
    items.reserve((size_t)nCases);
    for (int k : order)
        for (int c = 0; c < counts[k]; c++)
            items.push_back(MultiItem{k, (int)(caseBase[k] + c), stateBase[k] + (int64_t)c * grids[k]->sym.n});
    const int nItems = (int)items.size();
    std::vector<DevGrid> views(nGrids);
    for (int k = 0; k < nGrids; k++) views[k] = grids[k]->view;
    // slot layout
    const bool mixed = o.precision == GS_PREC_MIXED;
    const size_t t = mixed ? 4 : 8;
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    SlotArena arena{};
    size_t off = 0;
    arena.offLu = off; off += al((size_t)maxLu * t);
    arena.offPiv = off; off += al((size_t)maxM * t);
    arena.offY = off; off += al((size_t)maxM * t);
    arena.offZ = off; off += al(mixed ? (size_t)maxM * t : 0);
    arena.offRhs = off; off += al(mixed ? (size_t)maxM * 8 : 0);
    arena.offVm = off; off += al((size_t)maxN * 8);
    arena.offVa = off; off += al((size_t)maxN * 8);
    arena.offScal = off; off += al(sizeof(SlotScalars));
    arena.stride = off;
    // candidate CTA shapes and the CTAs each keeps resident
    int sms = 0;
    GS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    // autotuner candidates: CTA size x (top part in shared memory or every level in global memory)
    constexpr int kCand = 6;
    const int candThreads[kCand] = {1024, 512, 256, 1024, 512, 256};
    const int candTop[kCand] = {0, 0, 0, 1, 1, 1};
    size_t topBytes = 16;
    int maxLevels = 1;
    for (int k = 0; k < nGrids; k++)
        if (counts[k] > 0) {
            topBytes = std::max(topBytes, grids[k]->sym.top[mixed ? 1 : 0].bytes(t));
            maxLevels = std::max(maxLevels, grids[k]->sym.nLevels);
        }
    topBytes = (topBytes + 15) / 16 * 16;
    const size_t queueBytes = QueueBytes(maxLevels);
    int ctasOf[kCand];
    for (int q = 0; q < kCand; q++) {
        int occ = 0;
        const size_t sm = (candTop[q] ? topBytes : 0) + queueBytes;
        cudaError_t e = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_newton<float>, candThreads[q], sm)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_newton<double>, candThreads[q], sm);
        if (e != cudaSuccess) return SetErr(ctx, GS_ERR_CUDA, std::string("occupancy: ") + cudaGetErrorString(e));
        ctasOf[q] = std::max(1, occ) * sms;
    }
    // the arena holds the largest CTA count that fits in half the free memory
    size_t freeB = 0, totalB = 0;
    GS_CUDA(cudaMemGetInfo(&freeB, &totalB));
    const int maxSlots = (int)std::max<size_t>(1, std::min<size_t>((size_t)2048, (freeB / 2) / arena.stride));
    int slots = 1;
    for (int q = 0; q < kCand; q++) {
        ctasOf[q] = std::min(ctasOf[q], maxSlots);
        slots = std::max(slots, ctasOf[q]);
    }
    DevBuf dArena, dViews, dItems, dSample, dNext, dScale, dOut, dStatus, dIters, dMis, dVm, dVa, dSteps;
    GS_CUDA(dArena.alloc((size_t)slots * arena.stride));
    arena.base = dArena.as<char>();
    GS_CUDA(dViews.alloc(views.size() * sizeof(DevGrid)));
    GS_CUDA(cudaMemcpy(dViews.p, views.data(), views.size() * sizeof(DevGrid), cudaMemcpyHostToDevice));
    GS_CUDA(dItems.alloc(items.size() * sizeof(MultiItem)));
    GS_CUDA(cudaMemcpy(dItems.p, items.data(), items.size() * sizeof(MultiItem), cudaMemcpyHostToDevice));
    GS_CUDA(dNext.alloc(sizeof(int)));
    GS_CUDA(dSteps.alloc(sizeof(unsigned long long)));
    if (loadScale) {
        GS_CUDA(dScale.alloc((size_t)nStates * 8));
        GS_CUDA(cudaMemcpy(dScale.p, loadScale, (size_t)nStates * 8, cudaMemcpyHostToDevice));
    }
    if (outage) {
        GS_CUDA(dOut.alloc((size_t)nCases * 4));
        GS_CUDA(cudaMemcpy(dOut.p, outage, (size_t)nCases * 4, cudaMemcpyHostToDevice));
    }
    GS_CUDA(dStatus.alloc((size_t)nCases * 4));
    GS_CUDA(dIters.alloc((size_t)nCases * 4));
    GS_CUDA(dMis.alloc((size_t)nCases * 8));
    if (vmOut) GS_CUDA(dVm.alloc((size_t)nStates * 8));
    if (vaOut) GS_CUDA(dVa.alloc((size_t)nStates * 8));
    auto launch = [&](int q, const MultiItem* its, int nIts) {
        const size_t sm = (candTop[q] ? topBytes : 0) + queueBytes;
        const int qOff = candTop[q] ? (int)topBytes : 0;
        if (mixed)
            k_newton<float><<<ctasOf[q], candThreads[q], sm, st>>>(
                dViews.as<DevGrid>(), its, nIts, dNext.as<int>(), arena, dScale.as<double>(), dOut.as<int>(),
                dStatus.as<int>(), dIters.as<int>(), dMis.as<double>(), dVm.as<double>(), dVa.as<double>(), o.tolerance,
                o.diverge_limit_pu, o.max_iterations, dSteps.as<unsigned long long>(), candTop[q], qOff);
        else
            k_newton<double><<<ctasOf[q], candThreads[q], sm, st>>>(
                dViews.as<DevGrid>(), its, nIts, dNext.as<int>(), arena, dScale.as<double>(), dOut.as<int>(),
                dStatus.as<int>(), dIters.as<int>(), dMis.as<double>(), dVm.as<double>(), dVa.as<double>(), o.tolerance,
                o.diverge_limit_pu, o.max_iterations, dSteps.as<unsigned long long>(), candTop[q], qOff);
    };
    // autotuner: the CTA shape per set of grids (and precision), from timed trials on a sample of the items
    std::string key = mixed ? "m" : "d";
    for (int k = 0; k < nGrids; k++)
        if (counts[k] > 0) key += ":" + std::to_string((uintptr_t)grids[k]);
    int pick = -1;
    {
        std::lock_guard<std::mutex> l(ctx->mu);
        auto f = ctx->multiTune.find(key);
        if (f != ctx->multiTune.end()) pick = f->second;
    }
    float tuneMs = 0;
    const bool tuneNow = pick < 0;
    cudaEvent_t e0, e1;
    GS_CUDA(cudaEventCreate(&e0));
    GS_CUDA(cudaEventCreate(&e1));
    if (tuneNow) {
        const int nSample = std::min(nItems, 2 * slots);
        std::vector<MultiItem> sample(nSample);
        for (int j = 0; j < nSample; j++) sample[j] = items[(size_t)j * nItems / nSample];
        GS_CUDA(dSample.alloc(sample.size() * sizeof(MultiItem)));
        GS_CUDA(cudaMemcpy(dSample.p, sample.data(), sample.size() * sizeof(MultiItem), cudaMemcpyHostToDevice));
        float best = 0;
        for (int q = 0; q < kCand; q++) {
            cudaMemsetAsync(dNext.p, 0, sizeof(int), st);
            cudaEventRecord(e0, st);
            launch(q, dSample.as<MultiItem>(), nSample);
            cudaEventRecord(e1, st);
            GS_CUDA(cudaEventSynchronize(e1));
            GS_CUDA(cudaGetLastError());
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            tuneMs += ms;
            if (pick < 0 || ms < best) { best = ms; pick = q; }
        }
        std::lock_guard<std::mutex> l(ctx->mu);
        ctx->multiTune[key] = pick;
    }
    // the batch: reset of the item counter and the persistent launch, captured as one graph
    cudaGraph_t graph;
    cudaGraphExec_t exec = nullptr;
    GS_CUDA(cudaMemsetAsync(dSteps.p, 0, sizeof(unsigned long long), st));
    GS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(dNext.p, 0, sizeof(int), st);
    launch(pick, dItems.as<MultiItem>(), nItems);
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (ce == cudaSuccess) {
        ce = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
    }
    if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return SetErr(ctx, GS_ERR_CUDA, std::string("multi-grid graph: ") + cudaGetErrorString(ce));
    }
    cudaEventRecord(e0, st);
    ce = cudaGraphLaunch(exec, st);
    cudaEventRecord(e1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float ms = 0;
    if (ce == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaGraphExecDestroy(exec);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ce != cudaSuccess) return SetErr(ctx, GS_ERR_CUDA, std::string("multi-grid batch: ") + cudaGetErrorString(ce));
    if (status) GS_CUDA(cudaMemcpy(status, dStatus.p, (size_t)nCases * 4, cudaMemcpyDeviceToHost));
    if (iterations) GS_CUDA(cudaMemcpy(iterations, dIters.p, (size_t)nCases * 4, cudaMemcpyDeviceToHost));
    if (maxMismatch) GS_CUDA(cudaMemcpy(maxMismatch, dMis.p, (size_t)nCases * 8, cudaMemcpyDeviceToHost));
    if (vmOut) GS_CUDA(cudaMemcpy(vmOut, dVm.p, (size_t)nStates * 8, cudaMemcpyDeviceToHost));
    if (vaOut) GS_CUDA(cudaMemcpy(vaOut, dVa.p, (size_t)nStates * 8, cudaMemcpyDeviceToHost));
    if (stats) {
        unsigned long long steps = 0;
        GS_CUDA(cudaMemcpy(&steps, dSteps.p, sizeof(steps), cudaMemcpyDeviceToHost));
        stats->device_ms = ms;
        stats->tune_ms = tuneMs;
        stats->threads_per_cta = candThreads[pick];
        stats->shared_top = candTop[pick];
        stats->ctas = ctasOf[pick];
        stats->items = nItems;
        stats->tuned_now = tuneNow ? 1 : 0;
        stats->system_steps = (int64_t)steps;
    }
    return GS_OK;
}
