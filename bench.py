"""Benchmark: converged AC load flows per second of the batched N-1 branch-outage screen of a seeded
synthetic 10,000-bus grid (13,500 branches, 1,200 PV buses, 5,000 sampled non-islanding outages, every
outage a full Newton-Raphson solve warm-started from the base case, tolerance 1e-8 pu, at most 20
iterations, per-bus voltage limits), mixed precision (FP32 LU and triangular solves, FP64 mismatch,
update and residual refinement). The plain FP64 batched GPU solve of the same screen is reported beside
it (`fp64_value`).

A step is one complete screen of the outage set through the sharded screen (gridsim_b200.parallel.screen_sharded).
With --gpus N (torchrun, one process per GPU) the outage list is N sampled sets of 5,000 (N x 5,000 rows, seeds
0..N-1), dealt to the ranks by estimated cost (outage_costs / balanced_shards: about 5,000 per rank, weak
scaling), screened on each rank's GPU and all-gathered back into row order on every rank (no collective on the
data path); the device step time is the max over ranks, and `e2e` includes the gather and the merge.

`--impl reference` times the oracle (the C++ restatement of the reference's FP64 sparse
Gilbert-Peierls Newton-Raphson screen, one outage per host thread) on a bounded sample of the same
workload on all host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged AC load flows/sec (N-1, 10k-bus) mixed vs FP64 GPU; p99 serve latency"
UNIT = "load flows/s"
N_OUTAGES = 5000
GRID_SEED = 0


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait(timeout=10)

    def summary(self):
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload(rank=0, outages=N_OUTAGES, world=1):
    """The 10,000-bus grid and the outage rows of the whole job: `world` sampled sets of 5,000 non-islanding
    outages (seeds 0..world-1) one after the other; `outages` < 5,000 takes the first ones of each set (the small
    cases the committed profiles are captured on). `rank` is unused (every rank holds the whole list and screens
    its cost-balanced shard of it)."""
    from gridsim_b200 import synthetic
    del rank
    m = synthetic.config_grid(2, GRID_SEED)
    idx = np.concatenate([synthetic.outage_set(m, N_OUTAGES, GRID_SEED + r)[:outages] for r in range(world)])
    return m, idx.astype(np.int32)


def options(precision, timing=False):
    from gridsim_b200.engine import PowerFlowOptions
    return PowerFlowOptions(max_iterations=20, per_bus_voltage_limits=True, warm_start_from_base=True,
                            precision=precision, phase_timing=timing)


def cpu_sample(m, idx, threads, target_s=12.0):
    """The oracle on a bounded sample of the outage set: returns (solves/s, outages, seconds)."""
    import oracle
    o = options("fp64").to_c()
    probe = idx[: max(threads, 16)]
    t = time.time()
    oracle.screen(m, probe, o, threads=threads)
    dt = max(time.time() - t, 1e-3)
    k = int(min(len(idx), max(len(probe), len(probe) * target_s / dt)))
    sample = idx[:k]
    t = time.time()
    r = oracle.screen(m, sample, o, threads=threads)
    dt = time.time() - t
    conv = int((r["status"] == 0).sum())
    return conv / dt, k, dt


def cpu_single_thread(m, idx, count=6):
    """The oracle on one host thread: (solves/s, mean ms per outage solve) over `count` outages."""
    import oracle
    o = options("fp64").to_c()
    t = time.time()
    r = oracle.screen(m, idx[:count], o, threads=1)
    dt = max(time.time() - t, 1e-6)
    return int((r["status"] == 0).sum()) / dt, 1e3 * dt / count


# ---------------------------------------------------------------------------------------------
# Serving: Poisson arrivals of load-flow requests over the uneven grid population (64 synthetic grids, bus
# counts log-uniform in 100-25,000; each request the base case or one random non-islanding branch outage of a
# random grid, 50/50), answered by the request loop (gs_serve_*, mixed precision). Latency runs from the
# request's scheduled arrival to its result on the host.
SERVE_RATES = (100, 1000, 2000, 5000, 10000, 20000)
SERVE_HEADLINE_RATE = 1000
SERVE_SECONDS = 2.0


def serve_population(workers):
    from gridsim_b200 import synthetic
    grids = synthetic.uneven_population(64, 0, 100, 25000, workers=workers)
    outs = [synthetic.outage_set(m, None, 0) for m in grids]
    return grids, outs


def request_stream(outs, count, seed):
    from gridsim_b200.serving import REQUEST_DTYPE
    rng = np.random.default_rng(seed)
    arr = np.zeros(count, REQUEST_DTYPE)
    g = rng.integers(0, len(outs), count)
    lens = np.array([len(o) for o in outs])
    pick = (rng.random(count) * lens[g]).astype(np.int64)
    base = rng.random(count) < 0.5
    arr["grid"] = g
    arr["outage"] = [(-1 if base[k] or lens[g[k]] == 0 else int(outs[g[k]][pick[k]])) for k in range(count)]
    arr["tag"] = np.arange(count)
    return arr


def poisson_run(srv, reqs, rate, seed, drain_s=180.0):
    rng = np.random.default_rng(seed)
    n = len(reqs)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    lat = np.full(n, np.nan)
    status = np.full(n, -1)
    iters = np.zeros(n)
    delay = np.zeros(n)
    k = got = 0
    t0 = time.perf_counter()
    t_last = 0.0
    while got < n:
        now = time.perf_counter() - t0
        j = int(np.searchsorted(arrivals, now, side="right"))
        if j > k:
            delay[k:j] = (time.perf_counter() - t0) - arrivals[k:j]
            srv.submit(reqs[k:j])
            k = j
        res = srv.poll(timeout_ms=0)
        if res:
            t_last = time.perf_counter() - t0
            for r in res:
                lat[r.tag] = r.latency_ms + delay[r.tag] * 1e3
                status[r.tag] = r.status
                iters[r.tag] = r.iterations
            got += len(res)
        else:
            time.sleep(50e-6)
        if now > arrivals[-1] + drain_s:
            raise RuntimeError(f"serving at {rate} req/s: {n - got} requests unanswered")
    return {"rate_rps": rate, "requests": n, "offered_s": float(arrivals[-1]),
            "throughput_rps": n / max(t_last, 1e-9), "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "p999_ms": float(np.percentile(lat, 99.9)),
            "mean_ms": float(np.mean(lat)), "converged": float(np.mean(status == 0)),
            "mean_iterations": float(np.mean(iters))}


def batched_rps(ctx, grids, reqs, precision):
    """The same requests through the batched API, grouped by grid: outages as one N-1 screen per grid (warm
    start), base cases as one batch solve per grid. Wall time after one untimed pass."""
    from gridsim_b200.engine import ContingencyAnalysis, SparseNewtonRaphsonPowerFlow
    solvers = [SparseNewtonRaphsonPowerFlow(precision, ctx) for _ in grids]
    opt = options(precision)
    groups = []
    for g in range(len(grids)):
        sel = reqs[reqs["grid"] == g]["outage"]
        groups.append((np.ascontiguousarray(sel[sel >= 0], np.int32), int(np.sum(sel < 0))))

    def one_pass():
        for g, (m, (outs, nbase)) in enumerate(zip(grids, groups)):
            if len(outs):
                ContingencyAnalysis.screen_raw(m, outs, solvers[g], opt)
            if nbase:
                solvers[g].solve_batch(m, outage=np.full(nbase, -1, np.int32), options=opt)
    one_pass()
    t = time.perf_counter()
    one_pass()
    return len(reqs) / (time.perf_counter() - t)


STRESSED_MARGIN = 0.9


def run_stressed(ctx, outages, steps=2, warmup=1, check=True):
    """The same screen on the grid's stressed variant: the operating point at 0.9 (not 0.6) of the last solvable load
    level (same topology and outage set): outages take more Newton iterations, more of them fail and run to the cap.
    Both precisions, device-timed as the headline; a 48-outage check against the oracle."""
    from gridsim_b200 import synthetic
    from gridsim_b200.engine import ContingencyAnalysis, SparseNewtonRaphsonPowerFlow
    t = time.perf_counter()
    m = synthetic.config_grid(2, GRID_SEED, margin=STRESSED_MARGIN)
    gen_s = time.perf_counter() - t
    idx = synthetic.outage_set(m, N_OUTAGES, GRID_SEED)[:outages]
    out = {"workload": f"N-1 screen of the 10,000-bus grid stressed to {STRESSED_MARGIN} of its last solvable load "
                       f"level (load scale {m.meta.get('load_scale', 0):.4f}; the headline grid is at 0.6), "
                       f"{len(idx)} outages", "grid_build_s": gen_s}
    for prec in ("mixed", "fp64"):
        solver = SparseNewtonRaphsonPowerFlow(prec, ctx)
        opt = options(prec)
        for _ in range(warmup):
            ContingencyAnalysis.screen_raw(m, idx, solver, opt)
        dev = []
        for _ in range(steps):
            r = ContingencyAnalysis.screen_raw(m, idx, solver, opt)
            dev.append(r["device_ms"])
        conv = int((r["status"] == 0).sum())
        it = r["iterations"][r["status"] == 0]
        out[prec] = {"load_flows_per_s": conv / (float(np.mean(dev)) / 1e3), "ms_per_screen": float(np.mean(dev)),
                     "converged": conv, "not_converged": int(len(idx) - conv),
                     "mean_iterations_converged": float(it.mean()) if len(it) else None,
                     "newton_iterations": int(r["newton_iterations"])}
    out["mixed_over_fp64"] = out["mixed"]["load_flows_per_s"] / out["fp64"]["load_flows_per_s"]
    if check:
        import oracle
        sub = idx[:48]
        g = ContingencyAnalysis.screen_raw(m, sub, SparseNewtonRaphsonPowerFlow("mixed", ctx), options("mixed"),
                                           keep_states=True)
        o = oracle.screen(m, sub, options("fp64").to_c(), keep_states=True)
        cv = o["status"] == 0
        out["accuracy_vs_oracle"] = {
            "outages": int(len(sub)), "statuses_identical": bool(np.array_equal(g["status"], o["status"])),
            "max_dvm_pu": float(np.max(np.abs(g["vm"][cv] - o["vm"][cv]))),
            "max_dva_rad": float(np.max(np.abs(np.radians(g["va_deg"][cv] - o["va_deg"][cv])))),
            "violations_identical": bool(np.array_equal(g["viol_element"], o["viol_element"]))}
    return out


def run_uneven(ctx, grids, steps=3):
    """4,096 independent load flows (64 load scalings of each of the 64 grids: a global U(0.7, 1.3) times per-bus
    lognormal sigma 0.05), FP32 factor with FP64 mismatch, in one persistent graph-captured launch
    (gs_pf_solve_multi, CTA shape autotuned on the first call); beside it the same cases through the per-grid
    batched path (one gs_pf_solve_batch per grid) in both precisions."""
    from gridsim_b200 import synthetic
    from gridsim_b200.engine import PowerFlowOptions, SparseNewtonRaphsonPowerFlow, UnevenBatch
    scales = [synthetic.load_scalings(m, 64, k) for k, m in enumerate(grids)]
    counts = [64] * len(grids)
    out = {"workload": "4,096 load flows: 64 load scalings of each of 64 synthetic grids (100-25,000 buses)"}
    batch = UnevenBatch(grids, ctx)
    try:
        for prec in ("mixed", "fp64"):
            opt = PowerFlowOptions(precision=prec, max_iterations=20)
            r = batch.solve(counts, scales, None, opt)  # autotunes on this first call
            tune = dict(batch.stats)
            dev, wall = [], []
            for _ in range(steps):
                t = time.perf_counter()
                r = batch.solve(counts, scales, None, opt)
                wall.append(time.perf_counter() - t)
                dev.append(batch.stats["device_ms"])
            conv = int(sum(int((s == 0).sum()) for s in r["status"]))
            out[prec] = {"load_flows_per_s": conv / (float(np.median(dev)) / 1e3), "device_ms": float(np.median(dev)),
                         "e2e_load_flows_per_s": conv / float(np.median(wall)), "converged": conv,
                         "threads_per_cta": tune["threads_per_cta"], "ctas": tune["ctas"], "tune_ms": tune["tune_ms"],
                         "newton_steps": batch.stats["system_steps"]}
    finally:
        batch.close()
    for prec in ("mixed", "fp64"):
        opt = PowerFlowOptions(precision=prec, max_iterations=20)
        solvers = [SparseNewtonRaphsonPowerFlow(prec, ctx) for _ in grids]
        for g, m in enumerate(grids):
            solvers[g].solve_batch(m, load_scale=scales[g], options=opt)
        t = time.perf_counter()
        conv = 0
        for g, m in enumerate(grids):
            conv += int((solvers[g].solve_batch(m, load_scale=scales[g], options=opt)["status"] == 0).sum())
        out[f"per_grid_batched_{prec}_load_flows_per_s"] = conv / (time.perf_counter() - t)
    return out


def run_serving(ctx, grids, outs, gen_s):
    from gridsim_b200.serving import LoadFlowServer, drain
    srv = LoadFlowServer(options("mixed"), ctx)
    for m in grids:
        srv.add_grid(m)
    srv.start()
    try:
        warm = request_stream(outs, 2000, 99)
        srv.submit(warm)
        drain(srv, len(warm))
        runs = []
        for i, rate in enumerate(SERVE_RATES):
            reqs = request_stream(outs, int(max(200, rate * SERVE_SECONDS)), 1000 + i)
            runs.append(poisson_run(srv, reqs, rate, 2000 + i))
        st = srv.stats()
    finally:
        srv.close()
    ref_reqs = request_stream(outs, 20000, 77)
    out = {"population": f"64 synthetic grids, bus counts log-uniform 100-25,000 "
                         f"({sum(m.n_bus for m in grids):,} buses), built in {gen_s:.0f} s",
           "requests": "base case or one random non-islanding branch outage of a random grid (50/50)",
           "precision": "mixed", "max_slots_per_grid": 128, "slots_at_end": st["slots_total"],
           "slot_gb": st["slot_bytes"] / 1e9, "runs": runs,
           "batched_fp64_rps": batched_rps(ctx, grids, ref_reqs, "fp64"),
           "batched_mixed_rps": batched_rps(ctx, grids, ref_reqs, "mixed")}
    head = next(r for r in runs if r["rate_rps"] == SERVE_HEADLINE_RATE)
    return out, head


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    m, idx = workload(0)
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(args.warmup):
        cpu_sample(m, idx, threads, target_s=2.0)
    samples = []
    for _ in range(args.steps):
        v, k, dt = cpu_sample(m, idx, threads, target_s=10.0)
        vals.append(v)
        samples.append((k, dt))
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.median([s[1] for s in samples]) * 1e3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "N-1 screen, synthetic 10,000-bus grid, 5,000 non-islanding outages",
                       "n_bus": m.n_bus, "n_branch": m.n_branch, "outages": N_OUTAGES, "max_iterations": 20,
                       "tolerance": 1e-8},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{samples[0][0]} outages of the 5,000 per step, one outage per thread"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    from gridsim_b200.engine import ContingencyAnalysis, CudaContext, SparseNewtonRaphsonPowerFlow
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist_.init_process_group("nccl", timeout=timedelta(seconds=120))
        dist = dist_
    ctx = CudaContext(local)
    from gridsim_b200.parallel import balanced_shards, outage_costs, screen_sharded
    m, rows = workload(rank, args.outages, world)
    costs = outage_costs(m, rows) if world > 1 else None
    # this rank's shard (what its GPU screens); the accuracy check and the CPU legs run on it
    idx = rows[balanced_shards(costs, world)[rank]] if world > 1 else rows

    solvers = {}

    def screen(precision, timing=False):
        s = solvers.get(precision) or SparseNewtonRaphsonPowerFlow(precision, ctx)
        return s, ContingencyAnalysis.screen_raw(m, idx, s, options(precision, timing))

    def barrier():
        if dist:
            import torch
            dist.barrier()
            torch.cuda.synchronize()

    results = {}
    precs = ("mixed", "fp64") if args.precision == "both" else (args.precision,)
    for prec in precs:
        solver = SparseNewtonRaphsonPowerFlow(prec, ctx)
        solvers[prec] = solver
        opt = options(prec)
        own = {}
        # the grid's schedule (few-systems threshold, level-group cuts), autotuned on the rank's shard before the
        # warm-up (untimed; a 1,000-outage sample picked schedules that were no faster on the whole screen)
        tune = ContingencyAnalysis.tune_screen(m, idx, solver, opt) if not args.no_tune else None

        def screen_shard(mm, ii):
            own["r"] = ContingencyAnalysis.screen_raw(mm, ii, solver, opt)
            return own["r"]

        for _ in range(args.warmup):
            screen_sharded(m, rows, screen_shard, costs=costs)
        dev, wall, conv, launches = [], [], [], []
        sampler = ClockSampler(local)
        barrier()
        with sampler:
            for _ in range(args.steps):
                t = time.perf_counter()
                merged = screen_sharded(m, rows, screen_shard, costs=costs)
                wall.append(time.perf_counter() - t)
                r = own["r"]
                dev.append(r["device_ms"] / 1e3)
                conv.append(int((merged["status"] == 0).sum()))
                launches.append(int(r["kernel_launches"]))
        barrier()
        dev_t = float(np.sum(dev))
        wall_t = float(np.sum(wall))
        if dist:
            import torch
            t = torch.tensor([dev_t, wall_t], device=f"cuda:{local}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dev_t, wall_t = float(t[0]), float(t[1])
        # every rank holds the merged screen of all rows: its converged count is the job's
        total_conv = float(sum(conv))
        if tune is not None:
            # one untimed screen of the rank's shard under the default schedule, beside the tuned one's timed steps
            grid = solver.grid_for(m, opt)
            tuned = grid.schedule()
            grid.set_schedule()
            tune["default_screen_ms"] = float(ContingencyAnalysis.screen_raw(m, idx, solver, opt)["device_ms"])
            grid.set_schedule(**tuned)
            tune["tuned_screen_ms"] = float(np.mean(dev) * 1e3)
        results[prec] = dict(value=total_conv / dev_t, e2e=total_conv / wall_t, ms=dev_t / args.steps * 1e3,
                             wall_ms=wall_t / args.steps * 1e3, conv=conv[-1], launches=launches[-1],
                             clocks=sampler.summary(), last=r, schedule=tune)
    # phase timing (one extra untimed screen) for the roofline of the dominant kernel
    _, prof = screen("mixed", timing=True)
    peak, peak_kind = load_peaks()
    import ctypes
    from gridsim_b200 import _abi
    info = _abi.GridInfo()
    d = m.desc()
    _abi.load_library().gs_analyze_host(ctypes.byref(d), ctypes.byref(info))
    # the dominant kernel: the per-level factorisation of full-batch iterations (k_plevel<float, 0> launches and
    # the narrow-top k_ppersistent<float, 0>), its algorithmic bytes (J read + L, U written per system stepped)
    fb, fms = prof["level_factor_bytes"], prof["level_factor_ms"]
    achieved = fb / (fms / 1e3) / 1e9 if fms > 0 else None
    # measured DRAM bytes of one factorisation per system (ncu, committed under profiles/), against the same
    # unit as `achieved`'s numerator: bytes per system and full-batch factorisation
    traffic = None
    tf = os.path.join(ROOT, "profiles", "factor_traffic_per_system.json")
    if os.path.exists(tf):
        with open(tf) as fh:
            traffic = json.load(fh).get("bytes_per_system")
    # accuracy against the oracle on a small sample (untimed)
    acc = None
    if rank == 0 and not args.no_check:
        import oracle
        sub = idx[:48]
        from gridsim_b200.engine import ContingencyAnalysis as CA
        g = CA.screen_raw(m, sub, SparseNewtonRaphsonPowerFlow("mixed", ctx), options("mixed"), keep_states=True)
        o = oracle.screen(m, sub, options("fp64").to_c(), keep_states=True)
        cv = o["status"] == 0
        acc = {"outages": int(len(sub)), "flags_identical": bool(np.array_equal(g["status"] == 0, cv)),
               "max_dvm_pu": float(np.max(np.abs(g["vm"][cv] - o["vm"][cv]))),
               "max_dva_rad": float(np.max(np.abs(np.radians(g["va_deg"][cv] - o["va_deg"][cv])))),
               "violations_identical": bool(np.array_equal(g["viol_element"], o["viol_element"]) and
                                            np.array_equal(g["viol_kind"], o["viol_kind"]))}
    stressed = None
    if rank == 0 and world == 1 and not args.no_stress:
        stressed = run_stressed(ctx, args.outages, check=not args.no_check)
    serving, head, uneven = None, None, None
    if rank == 0 and not args.no_serve:
        t = time.perf_counter()
        grids, outs = serve_population(os.cpu_count() or 1)
        gen_s = time.perf_counter() - t
        uneven = run_uneven(ctx, grids)
        serving, head = run_serving(ctx, grids, outs, gen_s)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, k, dt = cpu_sample(m, idx, os.cpu_count() or 1)
        v1, ms1 = cpu_single_thread(m, idx)
        cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"{k} of the 5,000 outages ({dt:.1f} s), one outage per host thread",
               "one_thread_value": v1, "one_thread_ms_per_solve": ms1}
    if rank == 0:
        mx = results.get("mixed") or results["fp64"]
        fp = results.get("fp64") or {"value": None, "ms": None}
        last = mx["last"]
        out_bytes = len(idx) * (4 * 3 + 8 * 4) + 4 * (len(idx) + 1) + int(last["viol_ptr"][-1]) * 16
        line = {
            "metric": METRIC, "value": mx["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mx["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "N-1 screen, synthetic 10,000-bus grid, 5,000 non-islanding outages per GPU",
                       "n_bus": m.n_bus, "n_branch": m.n_branch, "n_pv": int(np.sum(m.bus_type == 2)),
                       "outages": int(len(rows)), "outages_rank0": int(len(idx)),
                       "sharding": "screen_sharded: rows dealt by estimated iterations (balanced_shards), "
                                   "results all-gathered in row order" if world > 1 else "screen_sharded, one rank",
                       "max_iterations": 20, "tolerance": 1e-8, "precision": "mixed" if "mixed" in results else "fp64",
                       "l2": "working set (LU of 5,000 systems, >1 GB) larger than L2",
                       "newton_iterations": int(last["newton_iterations"])},
            "fp64_value": fp["value"], "fp64_ms_per_step": fp["ms"],
            "mixed_over_fp64": (mx["value"] / fp["value"]) if fp["value"] and "mixed" in results else None,
            "converged_per_step": mx["conv"],
            "e2e": {"value": mx["e2e"], "unit": UNIT, "h2d_bytes_per_step": int(len(idx) * 4),
                    "d2h_bytes_per_step": int(out_bytes), "ms_per_step": mx["wall_ms"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "kernel": "k_plevel<float,0> + k_ppersistent<float,0>: fused static-pivot LU + forward "
                                   "substitution of full-batch iterations on the paired schedule",
                         "traffic_unit": "DRAM bytes per system and full-batch factorisation (ncu), beside "
                                         "bytes_per_system (algorithmic)",
                         "peak_source": peak_kind},
            "phase_ms": {"factor": prof["factor_ms"], "solve": prof["solve_ms"], "mismatch": prof["mismatch_ms"],
                         "other": prof["other_ms"], "few_systems_path": prof["tail_ms"],
                         "full_batch_factor": prof["level_factor_ms"]},
            "schedule": {p: results[p]["schedule"] for p in results},
            "cpu_baseline": cpu, "clocks": mx["clocks"], "gpu_launches": mx["launches"], "accuracy_vs_oracle": acc,
            "serve_p99_ms": head["p99_ms"] if head else None,
            "serve_rate_rps": SERVE_HEADLINE_RATE if head else None,
            "serving": serving,
            "uneven_batch": uneven,
            "stressed": stressed,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the grids' default schedule (no autotuning)")
    ap.add_argument("--no-stress", action="store_true", help="skip the screen of the stressed grid")
    ap.add_argument("--outages", type=int, default=N_OUTAGES,
                    help="screen the first K of the 5,000 sampled outages (small cases for profiling)")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="the screens to time (the headline is mixed; fp64 is its denominator)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
