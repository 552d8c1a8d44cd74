// gs_serve.cuh — the request loop (gs_serve_* of include/gridsim_b200.h). Part of gs_engine.cu's translation
// unit: it steps systems with the engine's kernels (mismatch + Jacobian fill, the per-system status test, the
// few-systems LU path, the FP64 refinement and the damped update).
//
// Continuous batching, one lane per registered grid. A lane owns a batch of C request slots (C <= 128, so
// that every stepping system gets its CTA or cluster of the few-systems walk in a single wave), its own stream and
// pinned staging. A tick is one Newton iteration of the lane's occupied slots, in two halves:
//   A: admit queued requests into free slots (k_admit: start voltages, Newton control), then mismatch +
//      Jacobian of every occupied slot, then the status test at each slot's own step count
//      (k_status_each lists the systems that stop); copy the counts, the stop list and the per-slot
//      results to pinned memory; event A.
//   B: copy out the solved states that were asked for (k_pack), then factor, solve and update the systems
//      still stepping; event B.
// Scheduler threads (each owning every k-th lane) poll their lanes' events and never block on the device: a request
// that arrives while its grid is mid-tick joins at the next tick, a finished request is answered as soon as half A
// shows it stopped (or, with a state, when half B has copied it), and the lanes of different grids overlap on the GPU.
// The reference's nearest host is sequential (src/GridSim.Cli/RpcCommand.cs:11-50: one request at a time).
#pragma once

#include <condition_variable>
#include <deque>

namespace gs {

// Start voltages and Newton control of newly admitted slots. admit[2c] = slot, admit[2c + 1] = outage.
// Grid (ceil(n / 8), ceil(nAdmit / 32)), block (32, 8).
__global__ void k_admit(DevGrid g, DevBatch b, const int* admit, int nAdmit, const double* baseVm, const double* baseVa) {
    const int c = blockIdx.y * 32 + threadIdx.x, i = blockIdx.x * 8 + threadIdx.y;
    if (c >= nAdmit || i >= g.n) return;
    const int s = admit[2 * c], o = admit[2 * c + 1];
    const size_t B = (size_t)b.B;
    const bool warm = baseVm && o >= 0;  // outages start from the solved base case, the base case from the case
    double vm = warm ? baseVm[i] : g.vm0[i];
    double va = warm ? baseVa[i] : g.va0[i];
    if (g.busType[i] != 1) vm = g.vm0[i];  // PV and slack magnitudes are set points (BuildBusSpec :467-469)
    if (g.busType[i] == 3) va = g.va0[i];
    b.vm[i * B + s] = vm;
    b.va[i * B + s] = va;
    if (i == 0) {
        b.maxMis[s] = 0ull;
        b.maxDx[s] = 0ull;
        b.startMis[s] = 0.0;
        b.finalMis[s] = NAN;
        b.status[s] = GS_PF_MAX_ITERATIONS;
        b.iters[s] = 0;
        b.convIters[s] = 0;
        if (b.refine) b.refine[s] = 0;
        b.flags[s] = 0;
        const_cast<int*>(b.outage)[s] = o;
        b.active[s] = 1;
    }
}

// Solved states of the listed slots, system-major: out[j * 2n + i] = Vm, out[j * 2n + n + i] = Va in degrees.
__global__ void k_pack(DevGrid g, DevBatch b, const int* list, int nPack, double* out) {
    const int j = blockIdx.y, i = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nPack || i >= g.n) return;
    const int s = list[j];
    const size_t B = (size_t)b.B, n = (size_t)g.n;
    out[j * 2 * n + i] = b.vm[i * B + s];
    out[j * 2 * n + n + i] = b.va[i * B + s] * (180.0 / 3.14159265358979323846);
}

namespace serve {

using ServeClock = std::chrono::steady_clock;

struct ServeTicket {
    uint64_t ticket = 0;
    gs_request req{};
    ServeClock::time_point submit, admit;
};

struct ServeResponse {
    gs_response r{};
    std::vector<double> state;
};

template <typename X>
struct PinnedBuf {
    X* p = nullptr;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() { if (p) cudaFreeHost(p); }
    cudaError_t alloc(size_t n) { return cudaMallocHost((void**)&p, std::max<size_t>(n, 1) * sizeof(X)); }
};

struct Lane {
    gs_grid* G = nullptr;
    int C = 0;           // slots (the batch's interleave stride), grown in steps of 32 up to Cmax as requests queue
    int Cmax = 0;
    double perSlot = 0;  // device bytes of one slot
    int stateSlots = 0;  // states copied out per tick
    bool warm = false;
    std::unique_ptr<Workspace> ws;
    std::vector<std::unique_ptr<Workspace>> retired;  // batches outgrown, freed when the loop is destroyed
    DevBuf admitD, doneD, stateD, baseVm, baseVa;
    cudaStream_t st = nullptr;
    cudaEvent_t evA = nullptr, evB = nullptr;
    PinnedBuf<int> hAdmit, hCounts, hDone, hStatus, hIters;
    PinnedBuf<double> hMis, hState;
    int phase = 0;  // 0 idle, 1 half A in flight, 2 half B in flight
    int nActive = 0, anyRefine = 0;
    std::vector<ServeTicket> slot;
    std::vector<int> freeSlots;
    std::deque<ServeTicket> pending;  // waiting for a free slot (scheduler thread only)
    std::vector<int> packWait;        // stopped, waiting for their state to be copied out
    std::vector<int> packing;         // states the half B in flight copies
    DevBatch batch{};
    ~Lane() {
        if (evA) cudaEventDestroy(evA);
        if (evB) cudaEventDestroy(evB);
        if (st) cudaStreamDestroy(st);
    }
    bool Busy() const { return phase != 0 || !pending.empty() || !packWait.empty(); }
};

}  // namespace serve
}  // namespace gs

struct gs_server {
    gs_ctx* ctx = nullptr;
    gs_serve_opts opts{};
    std::vector<std::unique_ptr<gs::serve::Lane>> lanes;
    double budget = 0, slotBytes = 0;
    std::vector<std::thread> threads;  // scheduler threads; thread t owns the lanes k with k % threads.size() == t
    int threadsRunning = 0;
    std::mutex mu;
    std::condition_variable cvIn, cvOut, cvDone;
    std::vector<std::deque<gs::serve::ServeTicket>> inbox;  // submitted requests, per scheduler thread
    std::deque<gs::serve::ServeResponse> done;
    uint64_t nextTicket = 1;
    bool batch = false;  // Q limits or the DC retry: queued requests answered in batches (AdvanceBatch)
    std::atomic<int> slotsTotal{0};  // slots of every lane
    bool started = false, stopping = false, abort = false, loopEnded = false, failed = false;
    int64_t submitted = 0, completed = 0;
    std::atomic<int64_t> ticks{0}, systemSteps{0};
    std::atomic<int> inFlight{0};
};

namespace gs {
namespace serve {

double MsBetween(ServeClock::time_point a, ServeClock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

void Post(gs_server* S, const Lane& L, int laneIndex, int s, const double* state) {
    const ServeTicket& t = L.slot[s];
    ServeResponse out;
    out.r.ticket = t.ticket;
    out.r.tag = t.req.tag;
    out.r.grid = laneIndex;
    out.r.outage = t.req.outage;
    out.r.status = L.hStatus.p[s];
    out.r.iterations = L.hIters.p[s];
    out.r.max_mismatch = L.hMis.p[s];
    const auto now = ServeClock::now();
    out.r.queue_ms = MsBetween(t.submit, t.admit);
    out.r.latency_ms = MsBetween(t.submit, now);
    out.r.state_offset = -1;
    if (state) out.state.assign(state, state + 2 * (size_t)L.G->sym.n);
    {
        std::lock_guard<std::mutex> l(S->mu);
        S->done.push_back(std::move(out));
        S->completed++;
    }
    S->inFlight--;
    S->cvOut.notify_all();
}

// Admission by device memory: a lane with more requests waiting than free slots grows, in steps of 32 slots to the
// width its systems in flight and waiting need (at most Cmax), if the request loop's device-memory budget still holds
// them (shared by every grid: memory goes to the grids that have requests). The systems in flight move into the wider
// batch (their voltages and Newton control; the Jacobian and right-hand side are rebuilt at the next half A). Called
// with the lane's stream idle (before half A). The outgrown batch is kept until the loop is destroyed: freeing device
// memory waits for the whole device, which would stall every other grid's iteration.
cudaError_t GrowLane(gs_server* S, Lane& L) {
    if (L.pending.size() <= L.freeSlots.size() || L.C >= L.Cmax) return cudaSuccess;
    const int want = L.C - (int)L.freeSlots.size() + (int)L.pending.size();
    const int C2 = std::min(L.Cmax, std::max(L.C + 32, (want + 31) / 32 * 32));
    {
        std::lock_guard<std::mutex> l(S->mu);
        const double more = C2 * L.perSlot;  // the new batch (the outgrown one stays allocated)
        if (S->slotBytes + more > S->budget) return cudaSuccess;  // no room: the requests wait for a free slot
        S->slotBytes += more;
    }
    const Symbolic& s = L.G->sym;
    auto nw = std::make_unique<Workspace>();
    if (EnsureWs(S->ctx, s, *nw, C2, S->opts.pf.precision, 0, false) != GS_OK) {
        std::lock_guard<std::mutex> l(S->mu);
        S->slotBytes -= C2 * L.perSlot;
        cudaGetLastError();
        return cudaSuccess;  // the allocation failed: stay at this width
    }
    cudaError_t e = cudaMemsetAsync(nw->active.p, 0, (size_t)C2 * sizeof(int), L.st);
    const DevBatch nb = MakeBatchWs(*nw, s.nLevels, C2, C2, false);
    std::vector<int2> pairs;
    for (int k = 0; k < L.C; k++) pairs.push_back(make_int2(k, k));  // every slot keeps its index (free ones inactive)
    DevBuf dp;
    if (e == cudaSuccess) e = dp.alloc(pairs.size() * sizeof(int2));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dp.p, pairs.data(), pairs.size() * sizeof(int2), cudaMemcpyHostToDevice, L.st);
    if (e == cudaSuccess) {
        k_move_listed<<<dim3((s.n + 7) / 8, (L.C + 31) / 32), dim3(32, 8), 0, L.st>>>(L.batch, nb, dp.as<int2>(), L.C, s.n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(L.st);
    if (e != cudaSuccess) return e;
    L.retired.push_back(std::move(L.ws));
    L.ws = std::move(nw);
    L.batch = nb;
    L.slot.resize(C2);
    for (int k = C2 - 1; k >= L.C; k--) L.freeSlots.push_back(k);
    S->slotsTotal += C2 - L.C;
    L.C = C2;
    return cudaSuccess;
}

template <typename T>
cudaError_t LaunchA(gs_server* S, Lane& L) {
    const gs_pf_opts& o = S->opts.pf;
    const DevGrid& g = L.G->view;
    if (cudaError_t e = GrowLane(S, L); e != cudaSuccess) return e;
    const DevBatch& b = L.batch;
    const dim3 blk8(32, 8);
    int nAdmit = 0;
    while (!L.freeSlots.empty() && !L.pending.empty()) {
        ServeTicket t = L.pending.front();
        L.pending.pop_front();
        const int s = L.freeSlots.back();
        L.freeSlots.pop_back();
        t.admit = ServeClock::now();
        L.slot[s] = t;
        L.hAdmit.p[2 * nAdmit] = s;
        L.hAdmit.p[2 * nAdmit + 1] = t.req.outage;
        nAdmit++;
    }
    if (nAdmit > 0) {
        cudaMemcpyAsync(L.admitD.p, L.hAdmit.p, (size_t)nAdmit * 2 * sizeof(int), cudaMemcpyHostToDevice, L.st);
        k_admit<<<dim3((g.n + 7) / 8, (nAdmit + 31) / 32), blk8, 0, L.st>>>(
            g, b, L.admitD.as<int>(), nAdmit, L.warm ? L.baseVm.as<double>() : nullptr, L.warm ? L.baseVa.as<double>() : nullptr);
    }
    cudaMemsetAsync(b.activeCount, 0, 2 * sizeof(int), L.st);
    cudaMemsetAsync(L.doneD.p, 0, sizeof(int), L.st);
    k_mismatch_jac<T><<<dim3((g.n + 7) / 8, L.C / 32), blk8, 0, L.st>>>(g, b, 1, nullptr, nullptr, nullptr, 0);
    k_status_each<<<(L.C + 255) / 256, 256, 0, L.st>>>(b, o.tolerance, o.diverge_limit_pu, o.max_iterations, L.doneD.as<int>());
    cudaMemcpyAsync(L.hCounts.p, b.activeCount, 2 * sizeof(int), cudaMemcpyDeviceToHost, L.st);
    cudaMemcpyAsync(L.hDone.p, L.doneD.p, (size_t)(1 + L.C) * sizeof(int), cudaMemcpyDeviceToHost, L.st);
    cudaMemcpyAsync(L.hStatus.p, b.status, (size_t)L.C * sizeof(int), cudaMemcpyDeviceToHost, L.st);
    cudaMemcpyAsync(L.hIters.p, b.iters, (size_t)L.C * sizeof(int), cudaMemcpyDeviceToHost, L.st);
    cudaMemcpyAsync(L.hMis.p, b.finalMis, (size_t)L.C * sizeof(double), cudaMemcpyDeviceToHost, L.st);
    cudaEventRecord(L.evA, L.st);
    L.phase = 1;
    return cudaGetLastError();
}

// After half A: answer the requests whose systems stopped (those that want their state wait for half B).
void AfterA(gs_server* S, Lane& L, int laneIndex) {
    L.nActive = L.hCounts.p[0];
    L.anyRefine = L.hCounts.p[1] > 0 ? 1 : 0;
    const int nd = L.hDone.p[0];
    for (int j = 0; j < nd; j++) {
        const int s = L.hDone.p[1 + j];
        if (L.slot[s].req.want_state) {
            L.packWait.push_back(s);
        } else {
            Post(S, L, laneIndex, s, nullptr);
            L.freeSlots.push_back(s);
        }
    }
}

template <typename T>
cudaError_t LaunchB(gs_server* S, Lane& L) {
    const DevGrid& g = L.G->view;
    const DevBatch& b = L.batch;
    const int n = g.n, m = g.m;
    const dim3 blk8(32, 8);
    const int refine = sizeof(T) < sizeof(double) ? L.anyRefine : 0;
    L.packing.clear();
    const int np = std::min<int>(L.stateSlots, (int)L.packWait.size());
    if (np > 0) {
        L.packing.assign(L.packWait.begin(), L.packWait.begin() + np);
        L.packWait.erase(L.packWait.begin(), L.packWait.begin() + np);
        for (int j = 0; j < np; j++) L.hAdmit.p[j] = L.packing[j];  // half A's copy of hAdmit has completed
        cudaMemcpyAsync(L.admitD.p, L.hAdmit.p, (size_t)np * sizeof(int), cudaMemcpyHostToDevice, L.st);
        k_pack<<<dim3((n + 127) / 128, np), 128, 0, L.st>>>(g, b, L.admitD.as<int>(), np, L.stateD.as<double>());
        cudaMemcpyAsync(L.hState.p, L.stateD.p, (size_t)np * 2 * n * sizeof(double), cudaMemcpyDeviceToHost, L.st);
    }
    const int na = L.nActive;
    if (na > 0) {
        cudaMemsetAsync(b.activeCount, 0, sizeof(int), L.st);
        k_collect_active<<<(L.C + 255) / 256, 256, 0, L.st>>>(b);
        FewSystemsSolve<T>(g, b, L.G->sym, na, L.G->tailSplit, refine != 0, L.st, nullptr, S->ctx->clusterOk,
                           L.G->paired);
        constexpr int rowsPerBlock = 512;
        k_dxmax<T><<<dim3((m + rowsPerBlock - 1) / rowsPerBlock, (na + 31) / 32), blk8, 0, L.st>>>(g, b, rowsPerBlock, refine,
                                                                                                b.activeList, na);
        k_update<T><<<dim3((n + 7) / 8, (na + 31) / 32), blk8, 0, L.st>>>(g, b, refine, b.activeList, na);
        S->ticks++;
        S->systemSteps += na;
    }
    cudaEventRecord(L.evB, L.st);
    L.phase = 2;
    return cudaGetLastError();
}

// After half B: answer the requests whose states were copied out.
void AfterB(gs_server* S, Lane& L, int laneIndex) {
    const size_t n2 = 2 * (size_t)L.G->sym.n;
    for (size_t j = 0; j < L.packing.size(); j++) {
        const int s = L.packing[j];
        Post(S, L, laneIndex, s, L.hState.p + j * n2);
        L.freeSlots.push_back(s);
    }
    L.packing.clear();
}

// One step of a lane's state machine; false when it is waiting on the device (or idle with nothing to do).
template <typename T>
bool Advance(gs_server* S, Lane& L, int laneIndex, cudaError_t* err) {
    *err = cudaSuccess;
    if (L.phase == 0) {
        if (!L.Busy()) return false;
        *err = LaunchA<T>(S, L);
        return true;
    }
    cudaEvent_t ev = L.phase == 1 ? L.evA : L.evB;
    const cudaError_t q = cudaEventQuery(ev);
    if (q == cudaErrorNotReady) return false;
    if (q != cudaSuccess) { *err = q; return true; }
    if (L.phase == 1) {
        AfterA(S, L, laneIndex);
        *err = LaunchB<T>(S, L);
    } else {
        AfterB(S, L, laneIndex);
        if (L.nActive > 0 || !L.pending.empty() || !L.packWait.empty()) *err = LaunchA<T>(S, L);
        else L.phase = 0;
    }
    return true;
}

// Batch mode (Q limits or the DC retry): a request's system changes between Newton passes (PV -> PQ switching, a
// second solve from DC angles), so it is not stepped in a slot; every request queued for the lane is answered by one
// gs_pf_solve_batch on the grid's own workspace, and requests that arrive meanwhile wait for the next batch. False
// when the lane has nothing queued; *rc is the call's status (the requests stay queued on a failure).
bool AdvanceBatch(gs_server* S, Lane& L, int laneIndex, int* rc) {
    *rc = GS_OK;
    if (L.pending.empty()) return false;
    std::vector<ServeTicket> take(L.pending.begin(), L.pending.end());
    L.pending.clear();
    const int count = (int)take.size();
    const size_t n = (size_t)L.G->sym.n;
    bool anyState = false;
    std::vector<int32_t> outage(count), status(count), iters(count);
    std::vector<double> mis(count);
    const auto admit = ServeClock::now();
    for (int k = 0; k < count; k++) {
        outage[k] = take[k].req.outage;
        anyState = anyState || take[k].req.want_state != 0;
        take[k].admit = admit;
    }
    std::vector<double> vm(anyState ? count * n : 0), va(anyState ? count * n : 0);
    *rc = gs_pf_solve_batch(L.G, count, nullptr, outage.data(), &S->opts.pf, status.data(), iters.data(), mis.data(),
                            anyState ? vm.data() : nullptr, anyState ? va.data() : nullptr);
    if (*rc != GS_OK) {
        L.pending.insert(L.pending.begin(), take.begin(), take.end());
        return true;
    }
    S->ticks++;
    S->systemSteps += count;
    const auto now = ServeClock::now();
    for (int k = 0; k < count; k++) {
        const ServeTicket& t = take[k];
        ServeResponse out;
        out.r.ticket = t.ticket;
        out.r.tag = t.req.tag;
        out.r.grid = laneIndex;
        out.r.outage = t.req.outage;
        out.r.status = status[k];
        out.r.iterations = iters[k];
        out.r.max_mismatch = mis[k];
        out.r.queue_ms = MsBetween(t.submit, t.admit);
        out.r.latency_ms = MsBetween(t.submit, now);
        out.r.state_offset = -1;
        if (t.req.want_state) {
            out.state.assign(vm.begin() + k * n, vm.begin() + (k + 1) * n);
            out.state.insert(out.state.end(), va.begin() + k * n, va.begin() + (k + 1) * n);
        }
        {
            std::lock_guard<std::mutex> l(S->mu);
            S->done.push_back(std::move(out));
            S->completed++;
        }
        S->inFlight--;
    }
    S->cvOut.notify_all();
    return true;
}

// Answer everything still outstanding with GS_PF_NOT_RUN (after a CUDA error stopped the loop).
void FailOutstanding(gs_server* S) {
    std::vector<ServeTicket> all;
    for (auto& lp : S->lanes) {
        Lane& L = *lp;
        std::vector<char> isFree(L.C, 0);
        for (int s : L.freeSlots) isFree[s] = 1;
        for (int s = 0; s < L.C; s++) if (!isFree[s]) all.push_back(L.slot[s]);
        for (auto& t : L.pending) all.push_back(t);
        L.pending.clear();
    }
    std::lock_guard<std::mutex> l(S->mu);
    for (auto& q : S->inbox) {
        for (auto& t : q) all.push_back(t);
        q.clear();
    }
    const auto now = ServeClock::now();
    for (auto& t : all) {
        ServeResponse out;
        out.r.ticket = t.ticket;
        out.r.tag = t.req.tag;
        out.r.grid = t.req.grid;
        out.r.outage = t.req.outage;
        out.r.status = GS_PF_NOT_RUN;
        out.r.max_mismatch = NAN;
        out.r.latency_ms = MsBetween(t.submit, now);
        out.r.state_offset = -1;
        S->done.push_back(std::move(out));
        S->completed++;
    }
    S->inFlight = 0;
}

// Scheduler thread `t` of `nt`: it owns the lanes k with k % nt == t, takes their requests from its inbox, and
// launches and polls their iterations. Several threads issue the lanes' launches in parallel (a lane's iteration is
// tens of launches, and with one thread their issue time, not the device, set the latency once many grids were busy).
// A CUDA error in any thread stops all of them; the last to leave answers what is outstanding.
void ServeLoop(gs_server* S, int t, int nt) {
    cudaSetDevice(S->ctx->device);
    const bool mixed = S->opts.pf.precision == GS_PREC_MIXED;
    std::vector<int> mine;
    for (int k = t; k < (int)S->lanes.size(); k += nt) mine.push_back(k);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            auto& in = S->inbox[t];
            while (!in.empty()) {
                ServeTicket tk = in.front();
                in.pop_front();
                S->lanes[tk.req.grid]->pending.push_back(tk);
            }
            if (S->abort || S->failed) break;
            bool busy = false;
            for (int k : mine) busy = busy || S->lanes[k]->Busy();
            if (!busy) {
                if (S->stopping) break;
                S->cvIn.wait(lk, [&] { return !S->inbox[t].empty() || S->stopping || S->abort || S->failed; });
                continue;
            }
        }
        bool progress = false;
        cudaError_t err = cudaSuccess;
        int rc = GS_OK;
        for (size_t q = 0; q < mine.size() && err == cudaSuccess && rc == GS_OK; q++) {
            const int k = mine[q];
            if (S->batch) progress |= AdvanceBatch(S, *S->lanes[k], k, &rc);
            else progress |= mixed ? Advance<float>(S, *S->lanes[k], k, &err) : Advance<double>(S, *S->lanes[k], k, &err);
        }
        if (err != cudaSuccess || rc != GS_OK) {
            if (err != cudaSuccess) SetErr(S->ctx, GS_ERR_CUDA, std::string("request loop: ") + cudaGetErrorString(err));
            {
                std::lock_guard<std::mutex> l(S->mu);
                S->failed = true;
            }
            S->cvIn.notify_all();
            break;
        }
        if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(5));
    }
    for (int k : mine)
        if (S->lanes[k]->st) cudaStreamSynchronize(S->lanes[k]->st);
    bool last = false, failed = false;
    {
        std::lock_guard<std::mutex> l(S->mu);
        last = --S->threadsRunning == 0;
        failed = S->failed;
    }
    if (!last) return;
    if (failed) FailOutstanding(S);  // every scheduler thread has left: the lanes are no one's now
    {
        std::lock_guard<std::mutex> l(S->mu);
        S->loopEnded = true;
    }
    S->cvDone.notify_all();
    S->cvOut.notify_all();
}

}  // namespace serve
}  // namespace gs

extern "C" {

int gs_serve_create(gs_ctx* ctx, const gs_serve_opts* opts, gs_server** out) {
    using namespace gs;
    using namespace gs::serve;
    if (!ctx || !opts || !out) return GS_ERR_INVALID_ARG;
    int rc = CheckOpts(ctx, &opts->pf);
    if (rc) return rc;
    if (opts->pf.flat_start) return SetErr(ctx, GS_ERR_UNSUPPORTED, "flat_start: pass a flat start in the descriptor");
    // Q limits and the DC retry (the options of the reference's rpc solve, src/GridSim.Cli/RpcCommand.cs:675-676):
    // answered in batches (AdvanceBatch), each request from the case's stored voltages as gs_pf_solve_batch starts them
    const bool batch = opts->pf.enforce_q_limits || opts->pf.retry_from_dc_start || opts->pf.partial_pivoting;
    if (batch && opts->pf.warm_start_from_base)
        return SetErr(ctx, GS_ERR_UNSUPPORTED, "warm_start_from_base with Q limits or the DC retry: not in the request loop");
    const int slots = opts->slots_per_grid ? opts->slots_per_grid : GS_SERVE_MAX_SLOTS;
    if (slots < 32 || slots > GS_SERVE_MAX_SLOTS || slots % 32)
        return SetErr(ctx, GS_ERR_INVALID_ARG, "slots_per_grid must be a multiple of 32 in [32, 128]");
    if (opts->scheduler_threads < 0) return SetErr(ctx, GS_ERR_INVALID_ARG, "scheduler_threads >= 0");
    if (opts->state_slots < 0 || opts->hbm_fraction < 0 || opts->hbm_fraction > 1)
        return SetErr(ctx, GS_ERR_INVALID_ARG, "state_slots >= 0 and hbm_fraction in [0, 1]");
    GS_CUDA(cudaSetDevice(ctx->device));
    size_t freeB = 0, totalB = 0;
    GS_CUDA(cudaMemGetInfo(&freeB, &totalB));
    auto* S = new gs_server();
    S->ctx = ctx;
    S->opts = *opts;
    S->batch = batch;
    S->opts.slots_per_grid = slots;
    if (S->opts.state_slots == 0) S->opts.state_slots = 16;
    S->budget = (opts->hbm_fraction > 0 ? opts->hbm_fraction : 0.5) * (double)freeB;
    *out = S;
    return GS_OK;
}

int gs_serve_add_grid(gs_server* S, gs_grid* G, int32_t* index) {
    using namespace gs;
    using namespace gs::serve;
    if (!S || !G || !index) return GS_ERR_INVALID_ARG;
    gs_ctx* ctx = S->ctx;
    if (G->ctx != ctx) return SetErr(ctx, GS_ERR_INVALID_ARG, "the grid belongs to another context");
    if (S->started) return SetErr(ctx, GS_ERR_STATE, "grids are added before gs_serve_start");
    GS_CUDA(cudaSetDevice(ctx->device));
    const gs_pf_opts& o = S->opts.pf;
    const Symbolic& s = G->sym;
    auto L = std::make_unique<Lane>();
    L->G = G;
    if (S->batch) {  // answered through gs_pf_solve_batch on the grid's own workspace: no slot batch
        *index = (int32_t)S->lanes.size();
        S->lanes.push_back(std::move(L));
        return GS_OK;
    }
    L->stateSlots = std::min(S->opts.state_slots, S->opts.slots_per_grid);
    const double per = (double)PerSystemBytes(s, o.precision);
    const double fixed = (double)L->stateSlots * 2.0 * s.n * 8.0 + 2.0 * s.n * 8.0;
    // every grid starts with 32 slots; it grows by 32 at a time (up to slots_per_grid) while its requests queue and
    // the budget holds the memory (GrowLane)
    const int C = 32;
    if (S->slotBytes + fixed + C * per > S->budget)
        return SetErr(ctx, GS_ERR_OOM, "the device memory budget of the request loop holds no more slots");
    L->C = C;
    L->Cmax = S->opts.slots_per_grid;
    L->perSlot = per;
    if (o.warm_start_from_base) {
        int st = 0, it = 0;
        double mis = 0;
        float ms = 0;
        int rc = SolveBase(G, o, &st, &it, &mis, &ms);
        if (rc) return rc;
        L->warm = st == GS_PF_CONVERGED;
    }
    GS_CUDA(L->baseVm.alloc((size_t)s.n * 8));
    GS_CUDA(L->baseVa.alloc((size_t)s.n * 8));
    if (L->warm) {
        GS_CUDA(cudaMemcpy(L->baseVm.p, G->ws.startVm.p, (size_t)s.n * 8, cudaMemcpyDeviceToDevice));
        GS_CUDA(cudaMemcpy(L->baseVa.p, G->ws.startVa.p, (size_t)s.n * 8, cudaMemcpyDeviceToDevice));
    }
    L->ws = std::make_unique<Workspace>();
    int rc = EnsureWs(ctx, s, *L->ws, C, o.precision, 0, false);
    if (rc) return rc;
    GS_CUDA(cudaMemset(L->ws->active.p, 0, (size_t)C * sizeof(int)));
    // per-slot staging sized for the widest the lane may grow to
    const int Cm = L->Cmax;
    GS_CUDA(L->admitD.alloc((size_t)2 * Cm * sizeof(int)));
    GS_CUDA(L->doneD.alloc((size_t)(1 + Cm) * sizeof(int)));
    GS_CUDA(L->stateD.alloc((size_t)L->stateSlots * 2 * s.n * sizeof(double)));
    GS_CUDA(L->hAdmit.alloc((size_t)2 * Cm));
    GS_CUDA(L->hCounts.alloc(4));
    GS_CUDA(L->hDone.alloc((size_t)1 + Cm));
    GS_CUDA(L->hStatus.alloc(Cm));
    GS_CUDA(L->hIters.alloc(Cm));
    GS_CUDA(L->hMis.alloc(Cm));
    GS_CUDA(L->hState.alloc((size_t)L->stateSlots * 2 * s.n));
    GS_CUDA(cudaStreamCreateWithFlags(&L->st, cudaStreamNonBlocking));
    GS_CUDA(cudaEventCreateWithFlags(&L->evA, cudaEventDisableTiming));
    GS_CUDA(cudaEventCreateWithFlags(&L->evB, cudaEventDisableTiming));
    L->batch = MakeBatchWs(*L->ws, s.nLevels, C, C, false);
    L->slot.resize(C);
    for (int k = C - 1; k >= 0; k--) L->freeSlots.push_back(k);
    S->slotBytes += fixed + C * per;
    S->slotsTotal += C;
    *index = (int32_t)S->lanes.size();
    S->lanes.push_back(std::move(L));
    return GS_OK;
}

int gs_serve_start(gs_server* S) {
    using namespace gs;
    using namespace gs::serve;
    if (!S) return GS_ERR_INVALID_ARG;
    if (S->started) return SetErr(S->ctx, GS_ERR_STATE, "the request loop is already running");
    if (S->lanes.empty()) return SetErr(S->ctx, GS_ERR_STATE, "no grid added");
    // scheduler threads: one per grid up to 8 (or as asked); the batch mode runs its solves on the context's one
    // stream, so it keeps one thread
    int nt = S->opts.scheduler_threads > 0 ? S->opts.scheduler_threads : 8;
    nt = std::max(1, std::min<int>(nt, (int)S->lanes.size()));
    if (S->batch) nt = 1;
    S->inbox.assign(nt, {});
    S->threadsRunning = nt;
    S->started = true;
    for (int t = 0; t < nt; t++) S->threads.emplace_back(ServeLoop, S, t, nt);
    return GS_OK;
}

int gs_serve_submit(gs_server* S, int32_t n, const gs_request* req, uint64_t* tickets) {
    using namespace gs;
    using namespace gs::serve;
    if (!S || n < 0 || (n > 0 && !req)) return GS_ERR_INVALID_ARG;
    for (int k = 0; k < n; k++) {
        const gs_request& r = req[k];
        if (r.grid < 0 || r.grid >= (int)S->lanes.size())
            return SetErr(S->ctx, GS_ERR_INVALID_ARG, "request " + std::to_string(k) + ": unknown grid " + std::to_string(r.grid));
        const HostGrid& h = S->lanes[r.grid]->G->host;
        if (r.outage < -1 || r.outage >= h.nbr || (r.outage >= 0 && !h.brOn[r.outage]))
            return SetErr(S->ctx, GS_ERR_INVALID_ARG,
                          "request " + std::to_string(k) + ": branch " + std::to_string(r.outage) + " is not an in-service branch");
    }
    const auto now = ServeClock::now();
    {
        std::lock_guard<std::mutex> l(S->mu);
        if (!S->started || S->stopping || S->failed || S->loopEnded)
            return SetErr(S->ctx, GS_ERR_STATE, "the request loop is not accepting requests");
        for (int k = 0; k < n; k++) {
            ServeTicket t;
            t.ticket = S->nextTicket++;
            t.req = req[k];
            t.submit = now;
            t.admit = now;
            if (tickets) tickets[k] = t.ticket;
            S->inbox[t.req.grid % S->inbox.size()].push_back(t);
        }
        S->submitted += n;
        S->inFlight += n;
    }
    S->cvIn.notify_all();
    return GS_OK;
}

int gs_serve_poll(gs_server* S, int32_t max, int32_t timeout_ms, gs_response* out, double* state, int64_t capacity,
                  int32_t* got) {
    using namespace gs;
    using namespace gs::serve;
    if (!S || max < 0 || (max > 0 && !out) || !got || capacity < 0 || (capacity > 0 && !state)) return GS_ERR_INVALID_ARG;
    *got = 0;
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->done.empty() && timeout_ms > 0)
        S->cvOut.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !S->done.empty() || S->loopEnded; });
    int64_t used = 0;
    while (*got < max && !S->done.empty()) {
        ServeResponse& r = S->done.front();
        if (!r.state.empty()) {
            if (used + (int64_t)r.state.size() > capacity) {
                if (*got == 0) return SetErr(S->ctx, GS_ERR_CAPACITY, "the state buffer cannot hold one solved state");
                break;
            }
            std::copy(r.state.begin(), r.state.end(), state + used);
            r.r.state_offset = used;
            used += (int64_t)r.state.size();
        }
        out[(*got)++] = r.r;
        S->done.pop_front();
    }
    return GS_OK;
}

int gs_serve_stats_get(gs_server* S, gs_serve_stats* st) {
    if (!S || !st) return GS_ERR_INVALID_ARG;
    std::memset(st, 0, sizeof(*st));
    std::lock_guard<std::mutex> l(S->mu);
    st->submitted = S->submitted;
    st->completed = S->completed;
    st->ticks = S->ticks;
    st->system_steps = S->systemSteps;
    st->grids = (int32_t)S->lanes.size();
    st->slots_total = S->slotsTotal;
    st->in_flight = S->inFlight;
    for (auto& q : S->inbox) st->queued += (int32_t)q.size();
    st->slot_bytes = S->slotBytes;
    st->failed = S->failed ? 1 : 0;
    return GS_OK;
}

int gs_serve_stop(gs_server* S, int32_t timeout_ms) {
    using namespace gs;
    using namespace gs::serve;
    if (!S) return GS_ERR_INVALID_ARG;
    if (!S->started) return GS_OK;
    int rc = GS_OK;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        S->stopping = true;
        S->cvIn.notify_all();
        if (!S->cvDone.wait_for(lk, std::chrono::milliseconds(std::max(timeout_ms, 0)), [&] { return S->loopEnded; })) {
            S->abort = true;  // the loop stops at its next pass; queued requests stay unanswered
            S->cvIn.notify_all();
            rc = SetErr(S->ctx, GS_ERR_TIMEOUT, "the request loop did not drain within the timeout");
        }
    }
    for (auto& th : S->threads)
        if (th.joinable()) th.join();
    S->threads.clear();
    S->started = false;
    return rc;
}

int gs_serve_destroy(gs_server* S) {
    if (!S) return GS_ERR_INVALID_ARG;
    if (S->started) gs_serve_stop(S, 60000);
    cudaSetDevice(S->ctx->device);
    delete S;
    return GS_OK;
}

}  // extern "C"
