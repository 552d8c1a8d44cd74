// GridSimB200.cs: the GridSim side of libgridsim_b200, the C ABI declared in gridsim_b200.h beside this file.
//
// Add the file to src/GridSim.Core. The project needs <AllowUnsafeBlocks>true</AllowUnsafeBlocks> (the fixed-size
// reserved fields of the option structures), and libgridsim_b200.so must sit where the runtime's native library
// probing finds it (beside the assembly, or on LD_LIBRARY_PATH). The file holds:
//
//   GsNative                       one P/Invoke declaration per entry point of gridsim_b200.h and its structures field
//                                  for field (LayoutKind.Sequential on x64 is the C layout);
//   GsContext, GsGrid              the device context (one per process) and a GridModel turned into a gs_grid_desc and
//                                  a device grid, cached per model instance (GridModel is immutable);
//   CudaSparseNewtonPowerFlow      IPowerFlowSolver (Abstractions/IPowerFlowSolver.cs:10-13) on gs_pf_solve;
//   CudaBatchedSparseLinearSolver  ISparseLinearSolver and IBatchedSparseLinearSolver (Abstractions/ISparseLinearSolver.cs:12-17,
//                                  IBatchedSparseLinearSolver.cs:19-37) on gs_sparse_solve_batch;
//   GsServer                       the request loop (gs_serve_*) for a resident host such as the rpc command's;
//   ContingencyAnalysis (partial)  ScreenBranchesCuda, ScreenBaseCaseCuda, ScreenOutagesCuda, ScreenNMinusKReportCuda and
//                                  ScreenElementOutagesCuda:
//                                  the screens of Analysis/ContingencyAnalysis.cs:306-344, :958-962, :944-950 and :1309-1437
//                                  as one device call each, labelled by the reference's own Label / LabelMany and
//                                  reported through its own NonConverged, so their rows read as the CPU screens' rows.
//
// Per-system outcomes never throw: they come back as statuses. A failed call maps GS_ERR_OOM to OutOfMemoryException,
// GS_ERR_INVALID_ARG to ArgumentException, GS_ERR_UNSUPPORTED to NotSupportedException, GS_ERR_TIMEOUT to
// TimeoutException and every other code to InvalidOperationException, each with the context's last error text.
// Models the library does not solve (HVDC links) are refused with NotSupportedException before any device call, so a
// caller can fall back to the CPU engines. Voltage-dependent (ZIP) loads are solved on the device.

namespace GridSim.Core.PowerFlow.B200
{
    using System;
    using System.Collections.Generic;
    using System.Runtime.CompilerServices;
    using System.Runtime.InteropServices;
    using System.Text;
    using GridSim.Core.Abstractions;
    using GridSim.Core.Model;
    using GridSim.Core.Numerics;

    /// <summary>The P/Invoke declarations of gridsim_b200.h (ABI version 1).</summary>
    public static unsafe class GsNative
    {
        public const string Lib = "gridsim_b200";
        public const int GS_ABI_VERSION = 2;

        // enum gs_status
        public const int GS_OK = 0, GS_ERR_INVALID_ARG = 1, GS_ERR_CUDA = 2, GS_ERR_OOM = 3, GS_ERR_NO_DEVICE = 4,
                         GS_ERR_TIMEOUT = 5, GS_ERR_STATE = 6, GS_ERR_UNSUPPORTED = 7, GS_ERR_INTERNAL = 8,
                         GS_ERR_CAPACITY = 9;
        // enum gs_pf_status: PowerFlowStatus in the same order, then the device-side outcomes
        public const int GS_PF_CONVERGED = 0, GS_PF_MAX_ITERATIONS = 1, GS_PF_NON_FINITE = 2, GS_PF_DIVERGED = 3,
                         GS_PF_SINGULAR_PIVOT = 4, GS_PF_TIMEOUT = 5, GS_PF_NOT_RUN = 6, GS_PF_UNSOLVABLE_PART = 7;
        // enum gs_post_fault_rating: PostFaultRating in the same order
        public const int GS_RATE_A = 0, GS_RATE_B = 1, GS_RATE_C = 2;
        // enum gs_precision
        public const int GS_PREC_FP64 = 0, GS_PREC_MIXED = 1;
        // enum gs_violation_kind: ContingencyViolationKind in the same order
        public const int GS_VIOL_BRANCH_OVERLOAD = 0, GS_VIOL_BOUNDARY_OVERLOAD = 1, GS_VIOL_UNDERVOLTAGE = 2,
                         GS_VIOL_OVERVOLTAGE = 3;
        // enum gs_outage_kind: OutageKind in the same order
        public const int GS_OUTAGE_BRANCH = 0, GS_OUTAGE_GENERATOR = 1, GS_OUTAGE_BUS = 2;
        // enum gs_ls_status
        public const int GS_LS_OK = 0, GS_LS_SINGULAR = 1, GS_LS_NON_FINITE_INPUT = 2, GS_LS_MALFORMED = 3;
        public const int GS_SERVE_MAX_SLOTS = 128;
        public const int GS_NOALLOC_MAX_SYSTEMS = 65536;

        [StructLayout(LayoutKind.Sequential)]
        public struct CtxOpts { public int ProbeTimeoutMs; public fixed int Reserved[7]; }

        [StructLayout(LayoutKind.Sequential)]
        public struct GridDesc
        {
            public int NBus, NGen, NBranch, Reserved0;
            public double BaseMva;
            public IntPtr BusId, BusType, Pd, Qd, Gs, Bs, Vm, VaDeg, VminPu, VmaxPu;   // int*, int*, double* ...
            public IntPtr GenBus, Pg, Qg, Vg, Qmin, Qmax, GenInService;                // int*, double* ..., byte*
            public IntPtr BrFrom, BrTo, R, X, B, Tap, ShiftDeg, RateA, BrInService;    // int*, int*, double* ..., byte*
            public IntPtr RateB, RateC;                                                // double*, may be zero
            public int NBoundary, Reserved1;
            public IntPtr BndPtr, BndBranch, BndDir, BndLimitMw;                       // CSR of (branch, +1/-1); MW
            public IntPtr Zip;                                                         // [6 n_bus] ZIP loads or 0
        }

        [StructLayout(LayoutKind.Sequential)]
        public struct PfOpts
        {
            public double Tolerance, DivergeLimitPu;
            public int MaxIterations, FlatStart, EnforceQLimits, RetryFromDcStart, PerBusVoltageLimits, Precision,
                       WarmStartFromBase, BatchWidth, PhaseTiming, PostFaultRating, MaxQLimitPasses, RevertQLimits,
                       PartialPivoting;
            public fixed int Reserved[3];
        }

        [StructLayout(LayoutKind.Sequential)]
        public struct PfResult
        {
            public int Status, Iterations;
            public double MaxMismatch;
            public IntPtr Vm, VaDeg, PInjMw, QInjMvar, LoadingPct, SfMva, StMva;       // caller-owned, may be zero
        }

        [StructLayout(LayoutKind.Sequential)]
        public struct N1Result
        {
            public IntPtr Status, Iterations, MaxMismatch, MinVm, MaxVm, MaxLoadingPct;  // [nOut]
            public IntPtr ViolPtr;                                                       // [nOut + 1]
            public int ViolCapacity, ViolCount;
            public IntPtr ViolKind, ViolElement, ViolValue;                              // [ViolCapacity]
            public IntPtr Vm, VaDeg;                                                     // [nOut * nBus] or zero
            public int BaseStatus, BaseIterations;
            public double DeviceMs;
            public int NSingularPivot, NBatches;
            public long KernelLaunches;
            public int NewtonIterations, NPartialPivot;
            public double FactorMs, SolveMs, MismatchMs, OtherMs, FactorBytes, LevelFactorMs, LevelFactorBytes, TailMs;
            public IntPtr Islanded, WorstBoundaryPct;                                    // byte*, double* [nOut] or zero
        }

        [StructLayout(LayoutKind.Sequential)]
        public struct GridInfo
        {
            public int NBus, NBranch, NPv, NPq, M, NnzY, NnzJ;
            public long NnzLu, LuFlops;
            public int NLevels;
            public fixed int Reserved[7];
        }

        // a grid's batched-solve schedule (no counterpart in the reference); gs_screen_tune picks it
        [StructLayout(LayoutKind.Sequential)]
        public struct Schedule
        {
            public int FactorCut, SolveCut, TailMax, Candidates;
            public double DefaultMs, TunedMs;
            public int SubtreeCut;
            public fixed int Reserved[3];
        }

        [StructLayout(LayoutKind.Sequential)]
        public struct MultiStats
        {
            public double DeviceMs, TuneMs;
            public int ThreadsPerCta, Ctas, Items, TunedNow;
            public long SystemSteps;
            public int SharedTop;
            public fixed int Reserved[7];
        }

        [StructLayout(LayoutKind.Sequential)]
        public struct ServeOpts
        {
            public PfOpts Pf;
            public int SlotsPerGrid, StateSlots;
            public double HbmFraction;
            public int SchedulerThreads;
            public fixed int Reserved[7];
        }

        [StructLayout(LayoutKind.Sequential)]
        public struct Request { public int Grid, Outage, WantState, Reserved; public ulong Tag; }

        [StructLayout(LayoutKind.Sequential)]
        public struct Response
        {
            public ulong Ticket, Tag;
            public int Grid, Outage, Status, Iterations;
            public double MaxMismatch, QueueMs, LatencyMs;
            public long StateOffset;
        }

        [StructLayout(LayoutKind.Sequential)]
        public struct ServeStats
        {
            public long Submitted, Completed, Ticks, SystemSteps;
            public int Grids, SlotsTotal, InFlight, Queued;
            public double SlotBytes;
            public int Failed;
            public fixed int Reserved[7];
        }

        // context
        [DllImport(Lib)] public static extern int gs_abi_version();
        [DllImport(Lib)] public static extern IntPtr gs_status_str(int status);
        [DllImport(Lib)] public static extern void gs_pf_opts_default(ref PfOpts o);
        [DllImport(Lib)] public static extern int gs_ctx_create(int device, ref CtxOpts opts, out IntPtr ctx);
        [DllImport(Lib)] public static extern int gs_ctx_destroy(IntPtr ctx);
        [DllImport(Lib)] public static extern int gs_last_error(IntPtr ctx, byte[] buf, UIntPtr len);

        // grids
        [DllImport(Lib)] public static extern int gs_grid_create(IntPtr ctx, ref GridDesc desc, out IntPtr grid);
        [DllImport(Lib)] public static extern int gs_grid_destroy(IntPtr grid);
        [DllImport(Lib)] public static extern int gs_grid_info_get(IntPtr grid, out GridInfo info);
        [DllImport(Lib)] public static extern int gs_analyze_host(ref GridDesc desc, out GridInfo info);
        [DllImport(Lib)] public static extern int gs_grid_schedule_get(IntPtr grid, out Schedule sched);
        [DllImport(Lib)] public static extern int gs_grid_schedule_set(IntPtr grid, ref Schedule sched);
        [DllImport(Lib)] public static extern int gs_screen_tune(IntPtr grid, int nOut, int[] branchIdx, ref PfOpts opts,
            out Schedule sched);

        // solves and screens
        [DllImport(Lib)] public static extern int gs_pf_solve(IntPtr grid, ref PfOpts opts, ref PfResult res);
        [DllImport(Lib)] public static extern int gs_pf_solve_batch(IntPtr grid, int count, double[]? loadScale,
            int[]? outage, ref PfOpts opts, int[] status, int[] iterations, double[] maxMismatch, double[]? vm,
            double[]? vaDeg);
        [DllImport(Lib)] public static extern int gs_n1_screen(IntPtr grid, int nOut, int[] branchIdx, ref PfOpts opts,
            ref N1Result res);
        [DllImport(Lib)] public static extern int gs_nk_screen(IntPtr grid, int nOut, int k, int[] branchSets,
            ref PfOpts opts, ref N1Result res);
        // kind: GS_OUTAGE_*; index: a branch, a position in GridDesc's generator arrays, or a bus position
        [DllImport(Lib)] public static extern int gs_element_screen(IntPtr grid, int nOut, int[] kind, int[] index,
            ref PfOpts opts, ref N1Result res);
        [DllImport(Lib)] public static extern int gs_outage_topology(ref GridDesc desc, double tolerance, int nOut,
            int[] branchIdx, byte[]? splits, byte[]? unsolvable);
        // status per system: GS_LS_*
        [DllImport(Lib)] public static extern int gs_sparse_solve_batch(IntPtr ctx, int count, int[] n, int[] rowPtr,
            int[] colIdx, double[] values, double[] rhs, double[] x, int[] status);
        [DllImport(Lib)] public static extern int gs_pf_mismatch_noalloc(IntPtr grid, int count, IntPtr dVm, IntPtr dVa,
            IntPtr dOutage, IntPtr dMaxMismatch);
        [DllImport(Lib)] public static extern int gs_pf_solve_multi(IntPtr ctx, int nGrids, IntPtr[] grids, int[] counts,
            double[]? loadScale, int[]? outage, ref PfOpts opts, int[] status, int[] iterations, double[] maxMismatch,
            double[]? vm, double[]? vaDeg, out MultiStats stats);

        // request loop
        [DllImport(Lib)] public static extern int gs_serve_create(IntPtr ctx, ref ServeOpts opts, out IntPtr server);
        [DllImport(Lib)] public static extern int gs_serve_add_grid(IntPtr server, IntPtr grid, out int gridIndex);
        [DllImport(Lib)] public static extern int gs_serve_start(IntPtr server);
        [DllImport(Lib)] public static extern int gs_serve_submit(IntPtr server, int n, Request[] req, ulong[]? tickets);
        [DllImport(Lib)] public static extern int gs_serve_poll(IntPtr server, int max, int timeoutMs,
            [Out] Response[] responses, double[]? state, long stateCapacity, out int got);
        [DllImport(Lib)] public static extern int gs_serve_stats_get(IntPtr server, out ServeStats stats);
        [DllImport(Lib)] public static extern int gs_serve_stop(IntPtr server, int timeoutMs);
        [DllImport(Lib)] public static extern int gs_serve_destroy(IntPtr server);

        /// <summary>The library's name for a call-level status.</summary>
        public static string StatusText(int status) => Marshal.PtrToStringAnsi(gs_status_str(status)) ?? $"status {status}";

        /// <summary>Throw the exception a failed call maps to (a no-op for GS_OK).</summary>
        public static void Check(int rc, IntPtr ctx, string call)
        {
            if (rc == GS_OK) return;
            string detail = "";
            if (ctx != IntPtr.Zero)
            {
                var buf = new byte[1024];
                if (gs_last_error(ctx, buf, (UIntPtr)buf.Length) == GS_OK)
                {
                    int len = Array.IndexOf(buf, (byte)0);
                    detail = Encoding.UTF8.GetString(buf, 0, len < 0 ? buf.Length : len);
                }
            }
            string msg = $"{call}: {StatusText(rc)}" + (detail.Length > 0 ? $" ({detail})" : "");
            Exception ex = rc switch
            {
                GS_ERR_OOM => new OutOfMemoryException(msg),
                GS_ERR_INVALID_ARG => new ArgumentException(msg),
                GS_ERR_UNSUPPORTED => new NotSupportedException(msg),
                GS_ERR_TIMEOUT => new TimeoutException(msg),
                _ => new InvalidOperationException(msg),
            };
            throw ex;
        }

        /// <summary>PowerFlowOptions (PowerFlow/PowerFlowOptions.cs:15-158) as gs_pf_opts. The reference's defaults
        /// are kept, Q limits and the DC retry included; <paramref name="precision"/> chooses the arithmetic of the
        /// linear step. FlatStart is not a flag of the call: the library takes a flat start through the descriptor's
        /// voltages (<see cref="GsGrid.For(GridModel, bool)"/>). Trace is not filled by the device path; Cancellation
        /// is honoured before the call.</summary>
        public static PfOpts Options(PowerFlowOptions? options, int precision)
        {
            var o = new PfOpts();
            gs_pf_opts_default(ref o);
            options ??= new PowerFlowOptions();
            options.Cancellation.ThrowIfCancellationRequested();
            o.Tolerance = options.Tolerance;
            o.DivergeLimitPu = options.DivergeLimitPu;
            o.MaxIterations = options.MaxIterations;
            o.EnforceQLimits = options.EnforceQLimits ? 1 : 0;
            o.MaxQLimitPasses = options.MaxQLimitPasses;
            o.RevertQLimits = options.RevertQLimits ? 1 : 0;
            o.RetryFromDcStart = options.RetryFromDcStart ? 1 : 0;
            o.PerBusVoltageLimits = options.PerBusVoltageLimits ? 1 : 0;
            o.PostFaultRating = (int)options.PostFaultRating;
            o.Precision = precision;
            return o;
        }
    }

    /// <summary>The arithmetic of the device's linear step; mismatch, update and convergence test are FP64 in both.</summary>
    public enum GsPrecision { Fp64 = GsNative.GS_PREC_FP64, Mixed = GsNative.GS_PREC_MIXED }

    /// <summary>One device context for the process (device 0 unless GRIDSIM_B200_DEVICE names another), opened on
    /// first use with the library's bounded probe and FP64 self-test, the part GpuContext plays for the ILGPU
    /// backends (GpuContext.cs:227-254).</summary>
    public static class GsContext
    {
        private static readonly Lazy<IntPtr> Ctx = new(Open, isThreadSafe: true);

        public static IntPtr Handle => Ctx.Value;

        /// <summary>True when the library loads, has this ABI version and opens a device.</summary>
        public static bool IsAvailable
        {
            get
            {
                try { return GsNative.gs_abi_version() == GsNative.GS_ABI_VERSION && Handle != IntPtr.Zero; }
                catch (DllNotFoundException) { return false; }
                catch (EntryPointNotFoundException) { return false; }
                catch (InvalidOperationException) { return false; }
                catch (TimeoutException) { return false; }
            }
        }

        private static IntPtr Open()
        {
            if (GsNative.gs_abi_version() != GsNative.GS_ABI_VERSION)
                throw new InvalidOperationException($"libgridsim_b200 has ABI version {GsNative.gs_abi_version()}, not {GsNative.GS_ABI_VERSION}.");
            int device = int.TryParse(Environment.GetEnvironmentVariable("GRIDSIM_B200_DEVICE"), out int d) ? d : 0;
            var opts = new GsNative.CtxOpts();
            GsNative.Check(GsNative.gs_ctx_create(device, ref opts, out IntPtr ctx), IntPtr.Zero, "gs_ctx_create");
            return ctx;   // held for the life of the process: every grid is destroyed before it
        }
    }

    /// <summary>A GridModel on the device: the gs_grid_desc built from it (bus ids resolved to positions, first
    /// occurrence, as the solvers key buses; the in-service generators of <see cref="GridModel.Generators"/>, so a
    /// generator index of the screens is the reference's; boundary member names resolved to their one branch) and the
    /// grid handle. One caller at a time uses a grid (<see cref="Sync"/>).</summary>
    public sealed class GsGrid : IDisposable
    {
        private static readonly ConditionalWeakTable<GridModel, GsGrid> Cache = new();
        private static readonly ConditionalWeakTable<GridModel, GsGrid> FlatCache = new();

        public GridModel Model { get; }
        public Handle Native { get; }
        public IReadOnlyDictionary<int, int> PositionOfBus { get; }
        public object Sync { get; } = new();

        /// <summary>The device grid of <paramref name="model"/>, built on first use and kept while the model lives;
        /// with <paramref name="flatStart"/>, the grid whose start voltages are PowerFlowOptions.FlatStart's.</summary>
        public static GsGrid For(GridModel model, bool flatStart = false)
        {
            ArgumentNullException.ThrowIfNull(model);
            return flatStart ? FlatCache.GetValue(model, m => new GsGrid(m, true)) : Cache.GetValue(model, m => new GsGrid(m, false));
        }

        /// <summary>A device grid of <paramref name="model"/> outside the cache, for a model used once: the caller
        /// disposes it (its device memory is released at once, not when the collector runs).</summary>
        public static GsGrid Uncached(GridModel model, bool flatStart = false)
        {
            ArgumentNullException.ThrowIfNull(model);
            return new GsGrid(model, flatStart);
        }

        public void Dispose() => Native.Dispose();

        private GsGrid(GridModel model, bool flatStart)
        {
            RequireSupported(model);
            Model = model;
            using var desc = new PinnedDesc(model, flatStart);
            PositionOfBus = desc.PositionOfBus;
            GsNative.GridDesc d = desc.Desc;
            GsNative.Check(GsNative.gs_grid_create(GsContext.Handle, ref d, out IntPtr g), GsContext.Handle, "gs_grid_create");
            Native = new Handle(g);
        }

        /// <summary>Refuse, before any device call, what the device path does not model.</summary>
        public static void RequireSupported(GridModel model)
        {
            if (model.HasCoupledDevices)
                throw new NotSupportedException("HVDC links are solved by HvdcCoupling on the CPU engines.");
        }

        /// <summary>The grid handle; gs_grid_destroy runs when the model and this wrapper are collected.</summary>
        public sealed class Handle : SafeHandle
        {
            public Handle(IntPtr h) : base(IntPtr.Zero, ownsHandle: true) { SetHandle(h); }
            public override bool IsInvalid => handle == IntPtr.Zero;
            protected override bool ReleaseHandle() => GsNative.gs_grid_destroy(handle) == GsNative.GS_OK;
        }

        /// <summary>A gs_grid_desc over pinned copies of a model's arrays; the library copies what it keeps during
        /// the call, so the pins end when this is disposed. With <c>flatStart</c> every bus that is not a reference
        /// bus starts at 1 pu and 0 degrees (a voltage-controlled bus with units still starts at their set point, a
        /// reference bus at its stored values: NewtonShell.cs:463-474).</summary>
        public sealed class PinnedDesc : IDisposable
        {
            private readonly List<GCHandle> _pins = new();
            public GsNative.GridDesc Desc;
            public Dictionary<int, int> PositionOfBus { get; } = new();

            public PinnedDesc(GridModel model, bool flatStart = false)
            {
                IReadOnlyList<Bus> buses = model.Buses;
                IReadOnlyList<Generator> gens = model.Generators;
                IReadOnlyList<Branch> branches = model.Branches;
                int n = buses.Count, ng = gens.Count, nb = branches.Count;
                for (int i = 0; i < n; i++) PositionOfBus.TryAdd(buses[i].Id, i);
                int Pos(int id, string what) => PositionOfBus.TryGetValue(id, out int p) ? p
                    : throw new ArgumentException($"{what} names bus {id}, which is not in the model.");

                var busId = new int[n]; var busType = new int[n];
                var pd = new double[n]; var qd = new double[n]; var gs = new double[n]; var bs = new double[n];
                var vm = new double[n]; var va = new double[n]; var vmin = new double[n]; var vmax = new double[n];
                for (int i = 0; i < n; i++)
                {
                    Bus b = buses[i];
                    busId[i] = b.Id;
                    busType[i] = b.Type switch { BusType.Slack => 3, BusType.Pv => 2, _ => 1 };
                    pd[i] = b.Pd; qd[i] = b.Qd; gs[i] = b.Gs; bs[i] = b.Bs;
                    bool flat = flatStart && b.Type != BusType.Slack;
                    vm[i] = flat ? 1.0 : b.Vm;
                    va[i] = flat ? 0.0 : b.VaDeg;
                    vmin[i] = b.VminPu ?? double.NaN; vmax[i] = b.VmaxPu ?? double.NaN;
                }
                var genBus = new int[ng];
                var pg = new double[ng]; var qg = new double[ng]; var vg = new double[ng];
                var qmin = new double[ng]; var qmax = new double[ng];
                for (int k = 0; k < ng; k++)
                {
                    Generator g = gens[k];
                    genBus[k] = Pos(g.Bus, $"generator {k}");
                    pg[k] = g.Pg; qg[k] = g.Qg; vg[k] = g.Vg; qmin[k] = g.Qmin; qmax[k] = g.Qmax;
                }
                var from = new int[nb]; var to = new int[nb];
                var r = new double[nb]; var x = new double[nb]; var bch = new double[nb];
                var tap = new double[nb]; var shift = new double[nb];
                var rateA = new double[nb]; var rateB = new double[nb]; var rateC = new double[nb];
                var inService = new byte[nb];
                for (int j = 0; j < nb; j++)
                {
                    Branch br = branches[j];
                    from[j] = Pos(br.From, $"branch {j}"); to[j] = Pos(br.To, $"branch {j}");
                    r[j] = br.R; x[j] = br.X; bch[j] = br.B; tap[j] = br.TapRatio; shift[j] = br.PhaseShiftDeg;
                    rateA[j] = br.RateAMva; rateB[j] = br.RateBMva; rateC[j] = br.RateCMva;
                    inService[j] = br.InService ? (byte)1 : (byte)0;
                }

                Desc = new GsNative.GridDesc
                {
                    NBus = n, NGen = ng, NBranch = nb, BaseMva = model.BaseMva,
                    BusId = Pin(busId), BusType = Pin(busType), Pd = Pin(pd), Qd = Pin(qd), Gs = Pin(gs), Bs = Pin(bs),
                    Vm = Pin(vm), VaDeg = Pin(va), VminPu = Pin(vmin), VmaxPu = Pin(vmax),
                    GenBus = Pin(genBus), Pg = Pin(pg), Qg = Pin(qg), Vg = Pin(vg), Qmin = Pin(qmin), Qmax = Pin(qmax),
                    GenInService = IntPtr.Zero,   // Generators holds the in-service units only
                    BrFrom = Pin(from), BrTo = Pin(to), R = Pin(r), X = Pin(x), B = Pin(bch), Tap = Pin(tap),
                    ShiftDeg = Pin(shift), RateA = Pin(rateA), BrInService = Pin(inService),
                    RateB = Pin(rateB), RateC = Pin(rateC),
                };

                IReadOnlyList<Boundary> bnd = model.Boundaries;
                if (bnd.Count > 0)
                {
                    Boundary.RequireResolvedBranchNames(model);   // every member names exactly one branch
                    var byName = new Dictionary<string, int>(StringComparer.Ordinal);
                    for (int j = 0; j < nb; j++)
                        if (!string.IsNullOrEmpty(branches[j].Name)) byName.TryAdd(branches[j].Name!, j);
                    var ptr = new int[bnd.Count + 1];
                    var member = new List<int>(); var dir = new List<int>();
                    var limit = new double[bnd.Count];
                    for (int q = 0; q < bnd.Count; q++)
                    {
                        foreach (BoundaryBranch m in bnd[q].Branches)
                        {
                            member.Add(byName[m.Branch]);
                            dir.Add(m.Direction);
                        }
                        ptr[q + 1] = member.Count;
                        limit[q] = bnd[q].LimitMw;
                    }
                    Desc.NBoundary = bnd.Count;
                    Desc.BndPtr = Pin(ptr);
                    Desc.BndBranch = Pin(member.ToArray());
                    Desc.BndDir = Pin(dir.ToArray());
                    Desc.BndLimitMw = Pin(limit);
                }

                // voltage-dependent loads (Bus.Zip): six coefficients a bus, constant power (0, 0, 1) where none varies
                bool anyZip = false;
                foreach (Bus b in buses) anyZip |= b.Zip is { VariesWithVoltage: true };
                if (anyZip)
                {
                    var zip = new double[6 * n];
                    for (int i = 0; i < n; i++)
                    {
                        ZipLoad z = buses[i].Zip is { VariesWithVoltage: true } v ? v : new ZipLoad();
                        zip[6 * i] = z.Ap; zip[6 * i + 1] = z.Bp; zip[6 * i + 2] = z.Cp;
                        zip[6 * i + 3] = z.Aq; zip[6 * i + 4] = z.Bq; zip[6 * i + 5] = z.Cq;
                    }
                    Desc.Zip = Pin(zip);
                }
            }

            private IntPtr Pin(Array a)
            {
                GCHandle h = GCHandle.Alloc(a, GCHandleType.Pinned);
                _pins.Add(h);
                return h.AddrOfPinnedObject();
            }

            public void Dispose()
            {
                foreach (GCHandle h in _pins) h.Free();
                _pins.Clear();
            }
        }
    }

    /// <summary>
    /// IPowerFlowSolver on the device: the sparse polar Newton-Raphson load flow of SparseNewtonRaphsonPowerFlow
    /// (PowerFlow/SparseNewtonRaphsonPowerFlow.cs), Q-limit passes and the DC-angle retry included, as one gs_pf_solve.
    /// The result is assembled as NewtonShell.AssembleResult does (PowerFlow/NewtonShell.cs:648-691): angles in degrees,
    /// injections in MW / MVAr, total loss as the sum of the injections, one LineFlow per branch of the model (zero for
    /// an out-of-service branch). SolvedBusTypes is left null and NewtonRetry NotTried: the C result carries neither.
    /// </summary>
    public sealed class CudaSparseNewtonPowerFlow : IPowerFlowSolver
    {
        public GsPrecision Precision { get; }

        public CudaSparseNewtonPowerFlow(GsPrecision precision = GsPrecision.Fp64) { Precision = precision; }

        public unsafe PowerFlowResult Solve(GridModel model, PowerFlowOptions? options = null)
        {
            GsGrid grid = GsGrid.For(model, options?.FlatStart == true);
            GsNative.PfOpts o = GsNative.Options(options, (int)Precision);
            int n = model.Buses.Count, nb = model.Branches.Count;
            var vm = new double[n]; var va = new double[n]; var p = new double[n]; var q = new double[n];
            var loading = new double[nb]; var sf = new double[2 * nb]; var st = new double[2 * nb];
            var res = new GsNative.PfResult();
            lock (grid.Sync)
            {
                fixed (double* pVm = vm, pVa = va, pP = p, pQ = q, pL = loading, pSf = sf, pSt = st)
                {
                    res.Vm = (IntPtr)pVm; res.VaDeg = (IntPtr)pVa; res.PInjMw = (IntPtr)pP; res.QInjMvar = (IntPtr)pQ;
                    res.LoadingPct = (IntPtr)pL; res.SfMva = (IntPtr)pSf; res.StMva = (IntPtr)pSt;
                    GsNative.Check(GsNative.gs_pf_solve(grid.Native.DangerousGetHandle(), ref o, ref res), GsContext.Handle,
                                   "gs_pf_solve");
                }
            }

            double lossP = 0, lossQ = 0;
            for (int i = 0; i < n; i++) { lossP += p[i]; lossQ += q[i]; }
            var busIds = new int[n];
            for (int i = 0; i < n; i++) busIds[i] = model.Buses[i].Id;
            var flows = new List<LineFlow>(nb);
            for (int j = 0; j < nb; j++)
            {
                Branch br = model.Branches[j];
                flows.Add(new LineFlow(br.From, br.To, sf[2 * j], sf[2 * j + 1], st[2 * j], st[2 * j + 1],
                    sf[2 * j] + st[2 * j], sf[2 * j + 1] + st[2 * j + 1], br.Name ?? "", br.RateAMva, loading[j]));
            }
            PowerFlowStatus status = StatusOf(res.Status);
            return new PowerFlowResult
            {
                Converged = status == PowerFlowStatus.Converged,
                Status = status,
                Iterations = res.Iterations,
                MaxMismatch = res.MaxMismatch,
                BusIds = busIds,
                Vm = vm,
                VaDeg = va,
                PInjMw = p,
                QInjMvar = q,
                TotalLossMw = lossP,
                TotalLossMvar = lossQ,
                LineFlows = flows,
            };
        }

        /// <summary>gs_pf_status as PowerFlowStatus: the first four are the same values; a collapsed static pivot and
        /// a provably unsolvable part end as the reference's solve does, MaxIterations (NewtonShell.cs:74-120).</summary>
        public static PowerFlowStatus StatusOf(int status) => status switch
        {
            GsNative.GS_PF_CONVERGED => PowerFlowStatus.Converged,
            GsNative.GS_PF_NON_FINITE => PowerFlowStatus.NonFinite,
            GsNative.GS_PF_DIVERGED => PowerFlowStatus.Diverged,
            GsNative.GS_PF_MAX_ITERATIONS or GsNative.GS_PF_SINGULAR_PIVOT or GsNative.GS_PF_UNSOLVABLE_PART
                => PowerFlowStatus.MaxIterations,
            GsNative.GS_PF_TIMEOUT => throw new TimeoutException("gs_pf_solve: a bounded device wait ran out."),
            _ => throw new InvalidOperationException($"gs_pf_solve: the system was not run (status {status})."),
        };
    }

    /// <summary>
    /// ISparseLinearSolver and IBatchedSparseLinearSolver on gs_sparse_solve_batch: systems of any sizes and patterns
    /// in one call, those sharing a pattern factorised together; the analysis of a pattern is kept on the context.
    /// Pivots are static on the diagonal of a minimum-degree order, after a row order that makes the diagonal
    /// structurally zero-free where it is not; a system whose diagonal pivot still collapses is reported singular
    /// (null) where the reference's row pivoting might have solved it.
    /// </summary>
    public sealed class CudaBatchedSparseLinearSolver : IBatchedSparseLinearSolver, ISparseLinearSolver
    {
        private readonly object _sync = new();

        public string Name => "cuda-b200 batched sparse LU";

        public double[]? Solve(CsrMatrix a, double[] b)
        {
            var errors = new Exception?[1];
            double[]?[] x = SolveBatch(new[] { a }, new[] { b }, errors);
            if (errors[0] is not null) throw errors[0]!;
            return x[0];
        }

        public double[]?[] SolveBatch(IReadOnlyList<CsrMatrix> matrices, IReadOnlyList<double[]> rhs, Exception?[] errors)
        {
            ArgumentNullException.ThrowIfNull(matrices);
            ArgumentNullException.ThrowIfNull(rhs);
            ArgumentNullException.ThrowIfNull(errors);
            int count = matrices.Count;
            if (rhs.Count != count || errors.Length != count)
                throw new ArgumentException($"{count} matrices, {rhs.Count} right-hand sides and {errors.Length} error slots.");
            int rows = 0, nnz = 0;
            for (int s = 0; s < count; s++)
            {
                CsrMatrix a = matrices[s] ?? throw new ArgumentException($"system {s} is null.");
                double[] b = rhs[s] ?? throw new ArgumentException($"right-hand side {s} is null.");
                if (b.Length != a.N) throw new ArgumentException($"system {s}: {a.N} rows but {b.Length} right-hand side values.");
                rows += a.N;
                nnz += a.RowPtr[a.N];
            }
            var n = new int[count]; var rowPtr = new int[rows + count]; var col = new int[nnz];
            var val = new double[nnz]; var bb = new double[rows]; var x = new double[rows]; var status = new int[count];
            int ro = 0, no = 0, bo = 0;
            for (int s = 0; s < count; s++)
            {
                CsrMatrix a = matrices[s];
                int e = a.RowPtr[a.N];
                n[s] = a.N;
                Array.Copy(a.RowPtr, 0, rowPtr, ro, a.N + 1);
                Array.Copy(a.ColIdx, 0, col, no, e);
                Array.Copy(a.Val, 0, val, no, e);
                Array.Copy(rhs[s], 0, bb, bo, a.N);
                ro += a.N + 1; no += e; bo += a.N;
            }
            lock (_sync)
                GsNative.Check(GsNative.gs_sparse_solve_batch(GsContext.Handle, count, n, rowPtr, col, val, bb, x, status),
                               GsContext.Handle, "gs_sparse_solve_batch");
            var result = new double[]?[count];
            bo = 0;
            for (int s = 0; s < count; s++)
            {
                switch (status[s])
                {
                    case GsNative.GS_LS_OK:
                        result[s] = new double[n[s]];
                        Array.Copy(x, bo, result[s]!, 0, n[s]);
                        break;
                    case GsNative.GS_LS_SINGULAR:
                        break;   // null: the caller takes its own fall-back path
                    case GsNative.GS_LS_NON_FINITE_INPUT:
                        errors[s] = new ArgumentException($"system {s}: the matrix or right-hand side holds a value that is not finite.");
                        break;
                    default:
                        errors[s] = new ArgumentException($"system {s}: the CSR structure is malformed.");
                        break;
                }
                bo += n[s];
            }
            return result;
        }
    }

    /// <summary>One answered request of <see cref="GsServer"/>: the caller's tag, the load flow's outcome and, when
    /// asked for, the solved state (Vm in pu, Va in degrees, in the model's bus order).</summary>
    public sealed record GsServedSolve(ulong Ticket, ulong Tag, int Grid, int Outage, PowerFlowStatus Status, int Iterations,
        double MaxMismatch, double QueueMs, double LatencyMs, double[]? Vm, double[]? VaDeg);

    /// <summary>
    /// The request loop (gs_serve_*) for a resident host such as the rpc command's (src/GridSim.Cli/RpcCommand.cs:667-700,
    /// which solves each held case with MaxIterations 100 and Q limits on): register the held cases, start, then submit
    /// and poll from any thread. With Q limits or the DC retry the loop answers in batches; no other solve may then use
    /// the process's device context while it runs.
    /// </summary>
    public sealed class GsServer : IDisposable
    {
        private IntPtr _server;
        private readonly List<int> _nBus = new();
        private readonly List<GsGrid> _grids = new();   // the grids must outlive the loop

        public GsServer(PowerFlowOptions? options = null, GsPrecision precision = GsPrecision.Fp64, int slotsPerGrid = 0)
        {
            var o = new GsNative.ServeOpts { Pf = GsNative.Options(options, (int)precision), SlotsPerGrid = slotsPerGrid };
            GsNative.Check(GsNative.gs_serve_create(GsContext.Handle, ref o, out _server), GsContext.Handle, "gs_serve_create");
        }

        /// <summary>Register a case (before <see cref="Start"/>); returns its grid index for requests.</summary>
        public int AddGrid(GridModel model, bool flatStart = false)
        {
            GsGrid grid = GsGrid.For(model, flatStart);
            GsNative.Check(GsNative.gs_serve_add_grid(_server, grid.Native.DangerousGetHandle(), out int index), GsContext.Handle,
                           "gs_serve_add_grid");
            _grids.Add(grid);
            _nBus.Add(model.Buses.Count);
            return index;
        }

        public void Start() => GsNative.Check(GsNative.gs_serve_start(_server), GsContext.Handle, "gs_serve_start");

        /// <summary>Queue requests: (grid, in-service branch index or -1 for the intact case, whether to return the
        /// state, the caller's tag). Returns their tickets.</summary>
        public ulong[] Submit(IReadOnlyList<(int Grid, int Outage, bool WantState, ulong Tag)> requests)
        {
            var req = new GsNative.Request[requests.Count];
            for (int k = 0; k < req.Length; k++)
                req[k] = new GsNative.Request
                {
                    Grid = requests[k].Grid, Outage = requests[k].Outage, WantState = requests[k].WantState ? 1 : 0,
                    Tag = requests[k].Tag,
                };
            var tickets = new ulong[req.Length];
            if (req.Length > 0)
                GsNative.Check(GsNative.gs_serve_submit(_server, req.Length, req, tickets), GsContext.Handle, "gs_serve_submit");
            return tickets;
        }

        /// <summary>Take up to <paramref name="max"/> answers, waiting up to <paramref name="timeoutMs"/> for the first.</summary>
        public IReadOnlyList<GsServedSolve> Poll(int max = 256, int timeoutMs = 0)
        {
            var resp = new GsNative.Response[max];
            long capacity = 0;
            foreach (int n in _nBus) capacity = Math.Max(capacity, 2L * n * max);
            var state = new double[capacity];
            GsNative.Check(GsNative.gs_serve_poll(_server, max, timeoutMs, resp, state, capacity, out int got), GsContext.Handle,
                           "gs_serve_poll");
            var answers = new List<GsServedSolve>(got);
            for (int k = 0; k < got; k++)
            {
                GsNative.Response r = resp[k];
                double[]? vm = null, va = null;
                if (r.StateOffset >= 0)
                {
                    int n = _nBus[r.Grid];
                    vm = new double[n];
                    va = new double[n];
                    Array.Copy(state, r.StateOffset, vm, 0, n);
                    Array.Copy(state, r.StateOffset + n, va, 0, n);
                }
                answers.Add(new GsServedSolve(r.Ticket, r.Tag, r.Grid, r.Outage, CudaSparseNewtonPowerFlow.StatusOf(r.Status),
                    r.Iterations, r.MaxMismatch, r.QueueMs, r.LatencyMs, vm, va));
            }
            return answers;
        }

        /// <summary>Finish every queued and running request, then stop the loop (their answers stay pollable).</summary>
        public void Stop(int timeoutMs = 60000) =>
            GsNative.Check(GsNative.gs_serve_stop(_server, timeoutMs), GsContext.Handle, "gs_serve_stop");

        public void Dispose()
        {
            if (_server == IntPtr.Zero) return;
            GsNative.gs_serve_destroy(_server);
            _server = IntPtr.Zero;
        }
    }
}

namespace GridSim.Core.Analysis
{
    using System;
    using System.Collections.Generic;
    using System.Globalization;
    using System.Linq;
    using GridSim.Core.Model;
    using GridSim.Core.PowerFlow;
    using GridSim.Core.PowerFlow.B200;

    /// <summary>The device screens: one library call per screen, rows built as ScreenStateCore builds them
    /// (ContingencyAnalysis.cs:1105-1240) from the call's per-outage summaries and violation lists.</summary>
    public static partial class ContingencyAnalysis
    {
        /// <summary>ScreenBranches / ScreenBranchesParallel / ScreenBranchesBatched (:306-344) as one gs_n1_screen:
        /// every in-service branch (or <paramref name="branchIndices"/>), results in that order.</summary>
        public static IReadOnlyList<ContingencyResult> ScreenBranchesCuda(GridModel model, PowerFlowOptions? options = null,
            IReadOnlyList<int>? branchIndices = null, GsPrecision precision = GsPrecision.Fp64)
        {
            ArgumentNullException.ThrowIfNull(model);
            int[] idx = branchIndices?.ToArray() ?? InServiceBranchIndices(model);
            if (branchIndices is not null) RequireInServiceOutages(model, idx, nameof(branchIndices));
            Boundary.RequireResolvedBranchNames(model);
            string[] labels = idx.Select(i => Label(model.Branches[i])).ToArray();
            return RunScreen(model, options, precision, labels, idx.Length,
                (IntPtr g, ref GsNative.PfOpts o, ref GsNative.N1Result r) => GsNative.gs_n1_screen(g, idx.Length, idx, ref o, ref r),
                "gs_n1_screen");
        }

        /// <summary>ScreenBaseCase (:958-962) on the device: the intact grid through the same classification.</summary>
        public static ContingencyResult ScreenBaseCaseCuda(GridModel model, PowerFlowOptions? options = null,
            GsPrecision precision = GsPrecision.Fp64)
        {
            ArgumentNullException.ThrowIfNull(model);
            Boundary.RequireResolvedBranchNames(model);
            var idx = new[] { -1 };
            return RunScreen(model, options, precision, new[] { BaseCaseLabel }, 1,
                (IntPtr g, ref GsNative.PfOpts o, ref GsNative.N1Result r) => GsNative.gs_n1_screen(g, 1, idx, ref o, ref r),
                "gs_n1_screen")[0];
        }

        /// <summary>ScreenOutage (:944-950) for many branch sets in one gs_nk_screen (each set's branches out together,
        /// at most sixteen per set), labelled by LabelMany as ScreenOutageCore labels them; the N-2 / N-k screens
        /// enumerate their combinations and hand them here.</summary>
        public static IReadOnlyList<ContingencyResult> ScreenOutagesCuda(GridModel model, IReadOnlyList<IReadOnlyList<int>> sets,
            PowerFlowOptions? options = null, GsPrecision precision = GsPrecision.Fp64)
        {
            ArgumentNullException.ThrowIfNull(model);
            ArgumentNullException.ThrowIfNull(sets);
            Boundary.RequireResolvedBranchNames(model);
            int k = Math.Max(1, sets.Count == 0 ? 1 : sets.Max(s => s.Count));
            var rows = new int[sets.Count * k];
            Array.Fill(rows, -1);
            var labels = new string[sets.Count];
            for (int j = 0; j < sets.Count; j++)
            {
                for (int t = 0; t < sets[j].Count; t++) rows[j * k + t] = sets[j][t];
                labels[j] = LabelMany(model, sets[j]);
            }
            int nOut = sets.Count;
            return RunScreen(model, options, precision, labels, nOut,
                (IntPtr g, ref GsNative.PfOpts o, ref GsNative.N1Result r) => GsNative.gs_nk_screen(g, nOut, k, rows, ref o, ref r),
                "gs_nk_screen");
        }

        /// <summary>ScreenNMinusKReport (:378-426) on the device: the single outages screened and ranked by the reference's
        /// own RankCandidates / StressScore (or every in-service branch when <paramref name="exhaustive"/>), its
        /// Combinations of k of them screened in one gs_nk_screen, the results worst first.</summary>
        public static NkScreenReport ScreenNMinusKReportCuda(GridModel model, int k, PowerFlowOptions? options = null,
            int candidateCount = DefaultCandidateCount, bool exhaustive = false, GsPrecision precision = GsPrecision.Fp64)
        {
            ArgumentNullException.ThrowIfNull(model);
            if (k < 1) throw new ArgumentOutOfRangeException(nameof(k), k, "contingency depth k must be >= 1");
            int[] live = InServiceBranchIndices(model);
            var none = Array.Empty<ContingencyResult>();
            if (k > live.Length) return new NkScreenReport(none, none) { Note = NkScreenReport.TooFewBranches(live.Length, k) };
            if (k == 1) return new NkScreenReport(ScreenBranchesCuda(model, options, null, precision), none);
            int[] candidates;
            IReadOnlyList<ContingencyResult> excluded = none;
            if (exhaustive)
            {
                candidates = live;
            }
            else
            {
                IReadOnlyList<ContingencyResult> single = ScreenBranchesCuda(model, options, null, precision);
                candidates = RankCandidates(single, candidateCount, k, out excluded).Select(i => live[i]).ToArray();
            }
            double comboCount = 1.0;
            for (int c = 0; c < k; c++) comboCount = comboCount * (candidates.Length - c) / (c + 1);
            if (comboCount > MaxCombinations)
                throw new ArgumentException(FormattableString.Invariant(
                    $"N-{k}: {candidates.Length} candidate branches give about {comboCount:G4} outage combinations, more than the {MaxCombinations} one screen takes; screen fewer candidates (a candidate count) or a smaller k."), nameof(k));
            var combos = new List<int[]>();
            Combinations(candidates, k, combos);
            IReadOnlyList<ContingencyResult> results =
                ScreenOutagesCuda(model, combos.Select(c => (IReadOnlyList<int>)c).ToList(), options, precision);
            return new NkScreenReport(results.OrderByDescending(StressScore).ToList(), excluded)
                { Note = NkScreenReport.TooFewCandidates(candidates.Length, excluded.Count, k) };
        }

        /// <summary>ScreenElementOutages (:1309-1320) with the reference-bus dispatch as one gs_element_screen: labels,
        /// lost load and generation and the notes as ScreenElementOutage gives them (:1343-1421). With governor droop or
        /// inertia, ShareLostPower moves the remaining units first; each such outage is then solved as the element
        /// outage of its own moved model (<see cref="MovedForSharing"/>), one device grid per outage.</summary>
        public static IReadOnlyList<ContingencyResult> ScreenElementOutagesCuda(GridModel model, IReadOnlyList<ElementOutage> outages,
            PowerFlowOptions? options = null, OutageDispatch dispatch = OutageDispatch.ReferenceBus,
            GsPrecision precision = GsPrecision.Fp64)
        {
            ArgumentNullException.ThrowIfNull(model);
            ArgumentNullException.ThrowIfNull(outages);
            Boundary.RequireResolvedBranchNames(model);
            int nOut = outages.Count;
            var kind = new int[nOut];
            var index = new int[nOut];
            var labels = new string[nOut];
            for (int j = 0; j < nOut; j++)
            {
                ElementOutage e = outages[j];
                kind[j] = (int)e.Kind;
                index[j] = e.Index;
                labels[j] = e.Kind switch
                {
                    OutageKind.Branch => Label(model.Branches[e.Index]),
                    OutageKind.Generator => "gen " + (string.IsNullOrEmpty(model.Generators[e.Index].Name)
                        ? $"{e.Index} at bus {model.Generators[e.Index].Bus}"
                        : $"{model.Generators[e.Index].Name} (bus {model.Generators[e.Index].Bus})"),
                    _ => "bus " + model.Buses[e.Index].Id
                         + (string.IsNullOrEmpty(model.Buses[e.Index].Name) ? "" : $" {model.Buses[e.Index].Name}"),
                };
            }
            IReadOnlyList<ContingencyResult> rows = RunScreen(model, options, precision, labels, nOut,
                (IntPtr g, ref GsNative.PfOpts o, ref GsNative.N1Result r) => GsNative.gs_element_screen(g, nOut, kind, index, ref o, ref r),
                "gs_element_screen");
            var results = new List<ContingencyResult>(nOut);
            for (int j = 0; j < nOut; j++)
            {
                ElementOutage e = outages[j];
                ContingencyResult row = rows[j];
                if (e.Kind == OutageKind.Generator)
                {
                    Generator gen = model.Generators[e.Index];
                    var gens = model.Generators.Where((_, i) => i != e.Index).ToList();
                    string? note = ReelectReference(model, model.Branches, gens, removedBusId: null, gen.Bus).Note;
                    row = row with { Kind = OutageKind.Generator, LostGenerationMw = gen.Pg, Note = note };
                }
                else if (e.Kind == OutageKind.Bus)
                {
                    Bus bus = model.Buses[e.Index];
                    var kept = model.Branches.Where(b => b.From != bus.Id && b.To != bus.Id).ToList();
                    var gens = model.Generators.Where(g => g.Bus != bus.Id).ToList();
                    double lostGen = model.Generators.Where(g => g.Bus == bus.Id).Sum(g => g.Pg);
                    string? note = ReelectReference(model, kept, gens, removedBusId: bus.Id, bus.Id).Note;
                    row = row with { Kind = OutageKind.Bus, LostLoadMw = bus.Pd, LostGenerationMw = lostGen, Note = note };
                }
                if (dispatch != OutageDispatch.ReferenceBus && e.Kind != OutageKind.Branch)
                {
                    GridModel? moved = MovedForSharing(model, e, dispatch, out string? shareNote);
                    if (moved is not null && !ReferenceEquals(moved, model))
                    {
                        using GsGrid own = GsGrid.Uncached(moved, options?.FlatStart == true);
                        int[] k1 = { kind[j] }, i1 = { index[j] };
                        ContingencyResult solved = RunScreen(model, options, precision, new[] { labels[j] }, 1,
                            (IntPtr g, ref GsNative.PfOpts o, ref GsNative.N1Result r) => GsNative.gs_element_screen(g, 1, k1, i1, ref o, ref r),
                            "gs_element_screen", own)[0];
                        row = solved with { Kind = row.Kind, LostLoadMw = row.LostLoadMw, LostGenerationMw = row.LostGenerationMw, Note = row.Note };
                    }
                    if (shareNote is not null) row = row with { Note = row.Note is null ? shareNote : row.Note + "; " + shareNote };
                }
                results.Add(row);
            }
            return results;
        }

        /// <summary>
        /// The model a shared-dispatch element outage is solved on (ScreenElementOutage, :1355-1421): ReelectReference
        /// and ShareLostPower, the reference's own, on the post-outage model, then written back into the full model, so
        /// that the device removes the unit or bus as usual. Its remaining units carry their shared output, and its
        /// reference is already re-elected (a removed reference bus is PQ), so the device does not re-elect it again by
        /// the moved output. Null when nothing is shared (no unit is left to take the reference: the reference-bus row
        /// stands); <paramref name="model"/> itself when no power was lost.
        /// </summary>
        private static GridModel? MovedForSharing(GridModel model, ElementOutage e, OutageDispatch dispatch, out string? shareNote)
        {
            shareNote = null;
            IReadOnlyList<Generator> all = model.Generators;
            var keep = new List<int>();   // positions in Generators of the units left
            IReadOnlyList<Branch> branches = model.Branches;
            double lost;
            int affected;
            int? removedBus = null;
            var island = new List<int>();
            if (e.Kind == OutageKind.Generator)
            {
                Generator gen = all[e.Index];
                for (int i = 0; i < all.Count; i++) if (i != e.Index) keep.Add(i);
                lost = gen.Pg;
                affected = gen.Bus;
                island.Add(gen.Bus);
            }
            else
            {
                Bus bus = model.Buses[e.Index];
                double lostGen = 0.0;
                for (int i = 0; i < all.Count; i++) { if (all[i].Bus == bus.Id) lostGen += all[i].Pg; else keep.Add(i); }
                lost = lostGen - bus.Pd;
                affected = bus.Id;
                removedBus = bus.Id;
                var kept = new List<Branch>(model.Branches.Count);
                foreach (Branch b in model.Branches)
                {
                    if (b.From != bus.Id && b.To != bus.Id) { kept.Add(b); continue; }
                    if (b.InService) island.Add(b.From == bus.Id ? b.To : b.From);
                }
                branches = kept;
            }
            var gens = new List<Generator>(keep.Count);
            foreach (int i in keep) gens.Add(all[i]);
            (IReadOnlyList<Bus>? buses, _, bool noUnitLeft) = ReelectReference(model, branches, gens, removedBusId: removedBus, affected);
            if (noUnitLeft) return null;
            IReadOnlyList<Bus> after = buses ?? model.Buses;
            var reducedBuses = new List<Bus>(after.Count);
            foreach (Bus b in after) if (removedBus is not int gone || b.Id != gone) reducedBuses.Add(b);
            GridModel reduced = model.CopyWith(buses: reducedBuses, generators: gens, branches: branches);
            (GridModel shared, string note) = ShareLostPower(reduced, lost, dispatch, island);
            shareNote = note;
            if (lost == 0.0) return model;
            var movedGens = new Generator[all.Count];
            for (int i = 0; i < all.Count; i++) movedGens[i] = all[i];
            for (int p = 0; p < keep.Count; p++) movedGens[keep[p]] = shared.Generators[p];
            var movedBuses = new List<Bus>(after.Count);
            foreach (Bus b in after)
                movedBuses.Add(removedBus is int r && b.Id == r && b.Type == BusType.Slack ? b with { Type = BusType.Pq } : b);
            return model.CopyWith(buses: movedBuses, generators: movedGens);
        }

        private delegate int ScreenCall(IntPtr grid, ref GsNative.PfOpts opts, ref GsNative.N1Result res);

        /// <summary>Run one screen call (again with a larger violation buffer when the library reports
        /// GS_ERR_CAPACITY) on <paramref name="grid"/> (default: the cached grid of <paramref name="model"/>) and build
        /// its rows, named from <paramref name="model"/>.</summary>
        private static unsafe IReadOnlyList<ContingencyResult> RunScreen(GridModel model, PowerFlowOptions? options,
            GsPrecision precision, string[] labels, int nOut, ScreenCall call, string name, GsGrid? grid = null)
        {
            if (nOut == 0) return Array.Empty<ContingencyResult>();
            grid ??= GsGrid.For(model, options?.FlatStart == true);
            GsNative.PfOpts o = GsNative.Options(options, (int)precision);
            var status = new int[nOut]; var iters = new int[nOut]; var mis = new double[nOut];
            var minVm = new double[nOut]; var maxVm = new double[nOut]; var maxLoad = new double[nOut];
            var worstBnd = new double[nOut]; var islanded = new byte[nOut]; var vptr = new int[nOut + 1];
            int cap = Math.Max(256, 16 * nOut);
            int[] vkind, vel; double[] vval;
            while (true)
            {
                vkind = new int[cap]; vel = new int[cap]; vval = new double[cap];
                var r = new GsNative.N1Result { ViolCapacity = cap };
                int rc;
                lock (grid.Sync)
                {
                    fixed (int* pS = status, pI = iters, pP = vptr, pK = vkind, pE = vel)
                    fixed (double* pM = mis, pLo = minVm, pHi = maxVm, pL = maxLoad, pB = worstBnd, pV = vval)
                    fixed (byte* pIs = islanded)
                    {
                        r.Status = (IntPtr)pS; r.Iterations = (IntPtr)pI; r.MaxMismatch = (IntPtr)pM;
                        r.MinVm = (IntPtr)pLo; r.MaxVm = (IntPtr)pHi; r.MaxLoadingPct = (IntPtr)pL;
                        r.ViolPtr = (IntPtr)pP; r.ViolKind = (IntPtr)pK; r.ViolElement = (IntPtr)pE; r.ViolValue = (IntPtr)pV;
                        r.Islanded = (IntPtr)pIs; r.WorstBoundaryPct = (IntPtr)pB;
                        rc = call(grid.Native.DangerousGetHandle(), ref o, ref r);
                    }
                }
                if (rc == GsNative.GS_ERR_CAPACITY) { cap = r.ViolCount + 64; continue; }
                GsNative.Check(rc, GsContext.Handle, name);
                break;
            }

            var results = new ContingencyResult[nOut];
            for (int j = 0; j < nOut; j++)
            {
                if (status[j] == GsNative.GS_PF_TIMEOUT)
                    throw new TimeoutException($"{name}: a bounded device wait ran out on '{labels[j]}'.");
                if (status[j] != GsNative.GS_PF_CONVERGED)
                {
                    results[j] = NonConverged(labels[j], islanded[j] != 0);
                    continue;
                }
                var violations = new List<string>();
                var details = new List<ContingencyViolation>();
                double worstUnder = double.PositiveInfinity, worstOver = double.NegativeInfinity;
                for (int q = vptr[j]; q < vptr[j + 1]; q++)
                {
                    double v = vval[q];
                    switch (vkind[q])
                    {
                        case GsNative.GS_VIOL_BRANCH_OVERLOAD:
                        {
                            Branch br = model.Branches[vel[q]];
                            string bl = string.IsNullOrWhiteSpace(br.Name) ? $"{br.From}-{br.To}" : br.Name!;
                            violations.Add(string.Create(CultureInfo.InvariantCulture, $"branch {bl} {v:F0}%"));
                            details.Add(new ContingencyViolation(ContingencyViolationKind.BranchOverload, vel[q], v, bl));
                            break;
                        }
                        case GsNative.GS_VIOL_BOUNDARY_OVERLOAD:
                        {
                            string bn = model.Boundaries[vel[q]].Name;
                            violations.Add(string.Create(CultureInfo.InvariantCulture, $"boundary {bn} {v:F0}%"));
                            details.Add(new ContingencyViolation(ContingencyViolationKind.BoundaryOverload, vel[q], v, bn));
                            break;
                        }
                        case GsNative.GS_VIOL_UNDERVOLTAGE:
                            details.Add(new ContingencyViolation(ContingencyViolationKind.Undervoltage, vel[q], v, ""));
                            worstUnder = Math.Min(worstUnder, v);
                            break;
                        default:
                            details.Add(new ContingencyViolation(ContingencyViolationKind.Overvoltage, vel[q], v, ""));
                            worstOver = Math.Max(worstOver, v);
                            break;
                    }
                }
                // one line for the lowest undervoltage and one for the highest overvoltage, after the branch and
                // boundary lines (:1213-1236)
                if (!double.IsPositiveInfinity(worstUnder))
                    violations.Add(string.Create(CultureInfo.InvariantCulture, $"undervoltage {worstUnder:F3} p.u."));
                if (!double.IsNegativeInfinity(worstOver))
                    violations.Add(string.Create(CultureInfo.InvariantCulture, $"overvoltage {worstOver:F3} p.u."));
                results[j] = new ContingencyResult(labels[j], true, maxLoad[j], worstBnd[j], minVm[j], maxVm[j], violations)
                    { Details = details };
            }
            return results;
        }
    }
}
