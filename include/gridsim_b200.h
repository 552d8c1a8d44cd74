/*
 * gridsim_b200.h — C ABI of the B200-native AC load-flow / N-1 contingency engine.
 *
 * This is the drop-in boundary for GridSim.Core's sparse Newton-Raphson load flow and its
 * N-1 branch-outage screen. Every entry point is `extern "C"`, takes plain pointers and sizes,
 * returns an int status (0 = GS_OK) and never throws across the boundary. Conventions follow
 * the reference's P/Invoke layer (src/GridSim.Gpu/RocmInterop.cs:115-134 int statuses,
 * :196-237 opaque IntPtr handles and caller-owned arrays).
 *
 * Ownership: the caller allocates every input and output array; the library never keeps a
 * caller pointer past the call that received it. Threading: a gs_ctx may be shared by threads
 * for create/destroy of grids; each gs_grid admits one caller at a time (the reference's
 * solvers are "one instance per thread", src/GridSim.Core/PowerFlow/CpuSparseLuSolver.cs:17-20).
 *
 * Reference interfaces replaced (paths relative to the GridSim source tree):
 *   IPowerFlowSolver.Solve              src/GridSim.Core/Abstractions/IPowerFlowSolver.cs:10-13
 *   ContingencyAnalysis.ScreenBranches* src/GridSim.Core/Analysis/ContingencyAnalysis.cs:306-344,
 *                                       src/GridSim.Core/Analysis/ContingencyAnalysis.Batched.cs:55-136
 *   ContingencyAnalysis.ScreenBaseCase  src/GridSim.Core/Analysis/ContingencyAnalysis.cs:958-962
 *   ISparseLinearSolver.Solve           src/GridSim.Core/Abstractions/ISparseLinearSolver.cs:12-17
 *   IBatchedSparseLinearSolver.SolveBatch src/GridSim.Core/Abstractions/IBatchedSparseLinearSolver.cs:19-37
 */
#ifndef GRIDSIM_B200_H
#define GRIDSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GS_ABI_VERSION 2

/* ---- call-level status codes ------------------------------------------------------------ */
enum gs_status {
    GS_OK = 0,
    GS_ERR_INVALID_ARG = 1, /* malformed call: null pointer, bad size, bad index (ArgumentException) */
    GS_ERR_CUDA = 2,        /* a CUDA runtime call failed; gs_last_error has the text           */
    GS_ERR_OOM = 3,         /* device allocation failed (RocmSparseLinearSolver.cs:297-331 kept OOM apart) */
    GS_ERR_NO_DEVICE = 4,   /* no usable CUDA device / driver probe failed or timed out          */
    GS_ERR_TIMEOUT = 5,     /* a bounded wait ran out                                            */
    GS_ERR_STATE = 6,       /* wrong call order (e.g. solve before analyze)                      */
    GS_ERR_UNSUPPORTED = 7, /* an option this build does not implement (named in gs_last_error)  */
    GS_ERR_INTERNAL = 8,
    GS_ERR_CAPACITY = 9     /* a caller-supplied output array is too small; the needed size is returned */
};

/* ---- per-system solve status: PowerFlowStatus (src/GridSim.Core/PowerFlow/PowerFlowResult.cs:5-22)
 *      in the same order, plus two device-side outcomes --------------------------------------- */
enum gs_pf_status {
    GS_PF_CONVERGED = 0,
    GS_PF_MAX_ITERATIONS = 1,
    GS_PF_NON_FINITE = 2,
    GS_PF_DIVERGED = 3,
    GS_PF_SINGULAR_PIVOT = 4, /* a static pivot collapsed below its floor: the step could not be taken
                                 (the reference reports this state as MaxIterations, NewtonShell.cs:74-120) */
    GS_PF_TIMEOUT = 5,
    GS_PF_NOT_RUN = 6,
    GS_PF_UNSOLVABLE_PART = 7 /* not solved: the outage leaves a connected part with no reference bus whose
                                 real-power balance no state can meet, so the solve could only end non-converged
                                 (ContingencyAnalysis.ProvablyUnsolvablePart, Analysis/ContingencyAnalysis.cs:1750-1830) */
};

/* Rating an outage state's branch loadings are judged against (PostFaultRating,
 * src/GridSim.Core/PowerFlow/PowerFlowOptions.cs:162-170): the base case always uses RateA; a branch whose
 * RateB / RateC is 0 falls back to RateA (ContingencyAnalysis.PostFaultLoadingPercent, :1273-1284). */
enum gs_post_fault_rating { GS_RATE_A = 0, GS_RATE_B = 1, GS_RATE_C = 2 };

/* Arithmetic of the linear step (Jacobian values, LU, triangular solves). Mismatch, update and
 * convergence test are always FP64. */
enum gs_precision { GS_PREC_FP64 = 0, GS_PREC_MIXED = 1 /* FP32 LU + solves, FP64 residual */ };

/* ContingencyViolationKind (src/GridSim.Core/Analysis/ContingencyAnalysis.cs:144-154), same order. */
enum gs_violation_kind {
    GS_VIOL_BRANCH_OVERLOAD = 0,
    GS_VIOL_BOUNDARY_OVERLOAD = 1,
    GS_VIOL_UNDERVOLTAGE = 2,
    GS_VIOL_OVERVOLTAGE = 3
};

typedef struct gs_ctx gs_ctx;
typedef struct gs_grid gs_grid;

/* ---- context ----------------------------------------------------------------------------- */
typedef struct gs_ctx_opts {
    int32_t probe_timeout_ms; /* bound on the device probe + FP64 self-test (GpuContext.cs:311-363); 0 = 10000 */
    int32_t reserved[7];
} gs_ctx_opts;

/* ---- grid description: the fields of GridModel the load flow reads (Model/Model.cs:20-35 Bus,
 *      :91-114 Generator, :253-275 Branch). Bus references are 0-based POSITIONS in the bus arrays,
 *      not bus ids (the reference resolves ids to positions first, SparseNewtonRaphsonPowerFlow.cs:76-78). */
typedef struct gs_grid_desc {
    int32_t n_bus;
    int32_t n_gen;
    int32_t n_branch;
    int32_t reserved0;
    double base_mva;
    /* buses [n_bus] */
    const int32_t *bus_id;   /* external id, the key of voltage violations */
    const int32_t *bus_type; /* 1 = PQ, 2 = PV, 3 = slack */
    const double *pd, *qd;   /* MW, MVAr */
    const double *gs, *bs;   /* MW / MVAr at 1 pu */
    const double *vm;        /* start / fixed magnitude, pu */
    const double *va_deg;    /* start / fixed angle, degrees */
    const double *vmin_pu;   /* own voltage limits; NaN = none; the array itself may be NULL */
    const double *vmax_pu;
    /* generators [n_gen] */
    const int32_t *gen_bus; /* bus position */
    const double *pg, *qg, *vg, *qmin, *qmax;
    const uint8_t *gen_in_service; /* NULL = all in service */
    /* branches [n_branch], in GridModel.Branches order */
    const int32_t *br_from, *br_to; /* bus positions */
    const double *r, *x, *b;        /* series R, X and total charging B, pu */
    const double *tap;              /* off-nominal ratio, 0 = 1 (AdmittanceStamp.cs:63-66) */
    const double *shift_deg;
    const double *rate_a;           /* MVA, 0 = unrated */
    const uint8_t *br_in_service;   /* NULL = all in service */
    const double *rate_b, *rate_c;  /* short-term / emergency MVA, 0 = not given; each array may be NULL */
    /* transmission boundaries (Boundary, Model/Model.cs:516-560), CSR: members bnd_ptr[q] .. bnd_ptr[q+1]-1 of
       boundary q are branch positions (the one branch each member's name resolves to) with direction +1 / -1;
       limit 0 = no limit authored (flow reported, never overloaded) */
    int32_t n_boundary;
    int32_t reserved1;
    const int32_t *bnd_ptr;         /* [n_boundary+1] */
    const int32_t *bnd_branch;      /* [bnd_ptr[n_boundary]] */
    const int32_t *bnd_dir;
    const double *bnd_limit_mw;     /* [n_boundary] */
    /* voltage-dependent (ZIP) loads (Bus.Zip / ZipLoad, Model/Model.cs:33,45-90): per bus Ap, Bp, Cp, Aq, Bq, Cq; the
       load drawn at V pu is Pd (Ap V^2 + Bp V + Cp), Qd (Aq V^2 + Bq V + Cq). A bus whose A and B terms are all 0 is
       constant power; NULL = every load constant power */
    const double *zip;              /* [6 * n_bus] */
} gs_grid_desc;

/* ---- options: PowerFlowOptions (src/GridSim.Core/PowerFlow/PowerFlowOptions.cs:15-158) ---- */
typedef struct gs_pf_opts {
    double tolerance;               /* pu, default 1e-8 */
    double diverge_limit_pu;        /* default 10; +inf turns the stop off */
    int32_t max_iterations;         /* default 30 (StudyOptions 100) */
    int32_t flat_start;             /* default 0 */
    int32_t enforce_q_limits;       /* PV->PQ switching passes (SparseNewtonRaphsonPowerFlow.cs:118-160); default 0
                                       here (the reference's default is on); the multi-grid batch and the
                                       request loop run it through batch solves */
    int32_t retry_from_dc_start;    /* solve a stalled case again from DC power-flow angles (NewtonShell.SolveWithRetry,
                                       NewtonShell.cs:227-268); default 0 here (the reference's default is on);
                                       the multi-grid batch and the request loop run it through batch solves */
    int32_t per_bus_voltage_limits; /* judge buses against their own vmin/vmax (VoltageLimits.cs:55-67) */
    int32_t precision;              /* enum gs_precision */
    int32_t warm_start_from_base;   /* screens: solve the intact grid first and start every outage from
                                       its solution (GridScenario.WithSolvedVoltages, Simulation/GridScenario.cs:35-52) */
    int32_t batch_width;            /* systems per device batch; 0 = choose from free HBM */
    int32_t phase_timing;           /* 1: time each phase with CUDA events (no graph replay) into the result */
    int32_t post_fault_rating;      /* enum gs_post_fault_rating, screens only; default GS_RATE_A */
    int32_t max_q_limit_passes;     /* cap on PV->PQ switching passes (MaxQLimitPasses); 0 = the default 100 */
    int32_t revert_q_limits;        /* RevertQLimits: a pinned bus may go back to PV within a switching pass; 0 */
    int32_t partial_pivoting;       /* 1: every Newton step of every system by the per-system sparse LU with row partial
                                       pivoting (the reference's SparseLuFactorization.Factor, FP64, one warp per
                                       system) instead of the batched static-pivot factorisation; 0 (default): that
                                       factorisation only for systems whose static pivot collapses */
    int32_t reserved[3];
} gs_pf_opts;

/* Fill `o` with the reference defaults (PowerFlowOptions()) plus precision = FP64. */
void gs_pf_opts_default(gs_pf_opts *o);

/* ---- single-solve result: PowerFlowResult (PowerFlow/PowerFlowResult.cs) -------------------- */
typedef struct gs_pf_result {
    int32_t status;       /* enum gs_pf_status */
    int32_t iterations;
    double max_mismatch;  /* pu */
    /* caller-owned arrays, each may be NULL */
    double *vm;           /* [n_bus] pu */
    double *va_deg;       /* [n_bus] degrees */
    double *p_inj_mw;     /* [n_bus] */
    double *q_inj_mvar;   /* [n_bus] */
    double *loading_pct;  /* [n_branch], 0 for an out-of-service or unrated branch */
    double *sf_mva;       /* [2*n_branch] from-end complex power (re, im) MW / MVAr */
    double *st_mva;       /* [2*n_branch] to-end complex power */
} gs_pf_result;

/* ---- N-1 screen result (ContingencyResult, Analysis/ContingencyAnalysis.cs:9-96, with Details
 *      as a CSR list of (kind, element, value) per outage) ----------------------------------- */
typedef struct gs_n1_result {
    /* per outage [n_out] */
    int32_t *status;
    int32_t *iterations;
    double *max_mismatch;
    double *min_vm, *max_vm;   /* 0 when not converged (ContingencyAnalysis.cs:1661-1662) */
    double *max_loading_pct;
    /* violation details, CSR: entries viol_ptr[k] .. viol_ptr[k+1]-1 belong to outage k */
    int32_t *viol_ptr;         /* [n_out+1] */
    int32_t viol_capacity;     /* length of the three arrays below */
    int32_t viol_count;        /* out: entries written (or needed, with GS_ERR_CAPACITY) */
    int32_t *viol_kind;        /* enum gs_violation_kind */
    int32_t *viol_element;     /* original branch index, or bus id */
    double *viol_value;        /* loading % or Vm pu */
    /* optional full states [n_out * n_bus], may be NULL */
    double *vm;
    double *va_deg;
    /* base case (ScreenBaseCase) when warm_start_from_base is set, else status GS_PF_NOT_RUN */
    int32_t base_status;
    int32_t base_iterations;
    /* device time of the screen, milliseconds (CUDA events): the base solve, the Newton batches, the retry,
     * and the classification and compaction of the results */
    double device_ms;
    int32_t n_singular_pivot;  /* systems whose static pivot failed and whose partial-pivoting re-solve failed too */
    int32_t n_batches;
    /* work and phase timing of the screen (phase times only with gs_pf_opts.phase_timing) */
    int64_t kernel_launches;   /* kernels this call launched */
    int32_t newton_iterations; /* Newton iterations of the largest batch (device loop trips) */
    int32_t n_partial_pivot;   /* systems solved again with row partial pivoting after a static pivot failed */
    double factor_ms;          /* fused factorisation + forward substitution */
    double solve_ms;           /* backward substitution (+ the refinement solves in mixed precision) */
    double mismatch_ms;        /* mismatch + Jacobian fill (+ residual) */
    double other_ms;           /* status, max |dx|, update */
    double factor_bytes;       /* algorithmic bytes of the factor phase (J read + L,U written), whole call */
    /* the factorisations of full-batch iterations alone (per-level launches + the narrow-top kernel) */
    double level_factor_ms;
    double level_factor_bytes;
    double tail_ms;            /* iterations on the few-systems path, all phases */
    /* per outage, each may be NULL */
    uint8_t *islanded;         /* 1 when the state did not converge and the outage split the network into more
                                  connected parts than the grid has (ContingencyAnalysis.Splits, :1665-1687) */
    double *worst_boundary_pct;/* highest boundary loading, 0 when not converged or no boundary is limited */
} gs_n1_result;

/* ---- context -------------------------------------------------------------------------------- */

/* Open `device`, run a bounded FP64 self-test (GpuContext.cs:227-254, probe bound :325-345). */
int gs_ctx_create(int device, const gs_ctx_opts *opts, gs_ctx **out);
int gs_ctx_destroy(gs_ctx *ctx);
/* Last error text of calls on this context (NUL-terminated, truncated to len). */
int gs_last_error(gs_ctx *ctx, char *buf, size_t len);
const char *gs_status_str(int status);
int gs_abi_version(void);

/* ---- grid ----------------------------------------------------------------------------------- */

/* Copy the grid in, build the base Y-bus (SparseNewtonRaphsonPowerFlow.BuildY :382-402 with
 * AdmittanceStamp.Branch, AdmittanceStamp.cs:35-76) and the shared symbolic analysis: equation
 * numbering (NewtonShell.EquationPositions, NewtonShell.cs:327-336), Jacobian superset pattern
 * (SparseNewtonRaphsonPowerFlow.BuildJacobianStructure :296-332), minimum-degree order
 * (Numerics/MinimumDegreeOrdering.cs:23-121), static-pivot LU pattern, level schedule; upload. */
int gs_grid_create(gs_ctx *ctx, const gs_grid_desc *desc, gs_grid **out);
int gs_grid_destroy(gs_grid *grid);

typedef struct gs_grid_info {
    int32_t n_bus, n_branch, n_pv, n_pq;
    int32_t m;          /* unknowns (n-1) + n_pq */
    int32_t nnz_y;
    int32_t nnz_j;      /* Jacobian superset pattern */
    int64_t nnz_lu;     /* L + U incl. diagonal, static-pivot pattern */
    int64_t lu_flops;   /* multiply-adds of one numeric factorisation */
    int32_t n_levels;   /* elimination-tree levels of the numeric schedule */
    int32_t reserved[7];
} gs_grid_info;
int gs_grid_info_get(gs_grid *grid, gs_grid_info *info);

/* Host-only: run the symbolic analysis of gs_grid_create without a device and report its sizes.
 * For planning batch sizes and for tests on machines without a GPU. */
int gs_analyze_host(const gs_grid_desc *desc, gs_grid_info *info);

/* ---- solves --------------------------------------------------------------------------------- */

/* IPowerFlowSolver.Solve on the intact grid (SparseNewtonRaphsonPowerFlow.Solve :48-54). */
int gs_pf_solve(gs_grid *grid, const gs_pf_opts *opts, gs_pf_result *res);

/* `count` independent load flows of the same grid in one device batch. Case k scales every bus's
 * Pd and Qd by load_scale[k*n_bus + i] (NULL = 1) and removes branch outage[k] (NULL or -1 = none).
 * Results go to vm/va_deg [count*n_bus] (may be NULL) and status/iterations/max_mismatch [count]. */
int gs_pf_solve_batch(gs_grid *grid, int32_t count, const double *load_scale, const int32_t *outage,
                      const gs_pf_opts *opts, int32_t *status, int32_t *iterations, double *max_mismatch,
                      double *vm, double *va_deg);

/* ContingencyAnalysis.ScreenBranches / ScreenBranchesParallel / ScreenBranchesBatched: one full
 * Newton solve per outaged branch (indices into the branch arrays; each must be in service; -1 is
 * the intact grid, ScreenBaseCase), then the ScreenStateCore classification
 * (ContingencyAnalysis.cs:1105-1238) on the device. Results are in the order of `branch_idx`.
 * Before any solve, a topology pass on the host finds the outages that leave a provably unsolvable part
 * (ScreenStateCore :1118-1127): those are reported GS_PF_UNSOLVABLE_PART and never reach the device.
 * With opts->post_fault_rating an outage state's loadings use RateB / RateC; limited boundaries add
 * GS_VIOL_BOUNDARY_OVERLOAD entries (element = boundary position) between the branch and voltage entries. */
int gs_n1_screen(gs_grid *grid, int32_t n_out, const int32_t *branch_idx, const gs_pf_opts *opts,
                 gs_n1_result *res);

/* Multi-branch outages (ScreenOutageCore over several indices, Analysis/ContingencyAnalysis.cs:1087-1097; the
 * N-k screens ScreenNMinusK :378-426 enumerate them): outage j takes out every branch branch_sets[j*k .. j*k+k-1]
 * that is not -1 (at most 16, distinct, in service; none = the intact grid). The Y cells each set touches get their
 * values without every branch of the set, summed in stamping order; everything else (topology pass, Newton solve,
 * retry, classification, result layout) is gs_n1_screen's, which is the k = 1 case. */
int gs_nk_screen(gs_grid *grid, int32_t n_out, int32_t k, const int32_t *branch_sets, const gs_pf_opts *opts,
                 gs_n1_result *res);

/* Single-element outages (ContingencyAnalysis.ScreenElementOutages / ScreenElementOutage,
 * Analysis/ContingencyAnalysis.cs:1309-1437): outage j takes out the branch, the generator (a position in the
 * generator arrays; the unit must be in service) or the bus (a position in the bus arrays) index[j] of kind[j].
 * A generator outage loses the unit's output, picked up by the reference bus; a PV bus left with no unit is solved
 * as PQ. A bus outage removes the bus with every branch touching it, its units and its load. When the outage takes
 * the reference bus or its last unit, the reference moves to the bus of the largest remaining unit by |Pg| in the
 * part the reference served (ReelectReference :1440-1488); with no unit there, the outage is reported
 * GS_PF_UNSOLVABLE_PART. These run on the grid analysed with every bus's P and Q rows (identity rows where a bus is
 * PV, the reference or removed in a system). Results as gs_n1_screen; a removed bus is left out of Vmin / Vmax and
 * of the voltage violations, its vm / va_deg entries are the start values. This call is the reference-bus dispatch
 * (OutageDispatch.ReferenceBus, the default). The shared dispatches (GovernorDroop, Inertia: ShareLostPower
 * :1509-1579) are the same call on a descriptor whose remaining units carry their shared output and whose reference
 * is already re-elected (a removed reference bus given as PQ); the host builds it per outage. */
enum gs_outage_kind { GS_OUTAGE_BRANCH = 0, GS_OUTAGE_GENERATOR = 1, GS_OUTAGE_BUS = 2 };
int gs_element_screen(gs_grid *grid, int32_t n_out, const int32_t *kind, const int32_t *index, const gs_pf_opts *opts,
                      gs_n1_result *res);

/* ---- batched sparse linear solve: ISparseLinearSolver.Solve (Abstractions/ISparseLinearSolver.cs:12-17) and
 *      IBatchedSparseLinearSolver.SolveBatch (Abstractions/IBatchedSparseLinearSolver.cs:19-37) ----------------
 * `count` square systems A_s x_s = b_s in FP64, of any sizes and patterns, in CSR, concatenated system after
 * system: n[s] rows; row_ptr holds n[s]+1 offsets per system (each block starting at 0); col_idx and values hold
 * row_ptr[n[s]] entries per system; rhs and x hold n[s] values per system. Systems that share a pattern are
 * factorised together on the device: static diagonal pivots on a minimum-degree order of A + A^T, after a row order
 * that makes the diagonal structurally zero-free where it is not (a maximum transversal; the reference
 * orders the same pattern, SparseLuFactorization.cs:69-195, but pivots by rows); the analysis of a pattern is kept
 * on the context for later calls, as CpuSparseLuSolver caches its ordering (CpuSparseLuSolver.cs:22-48). The inputs
 * are not modified. A system that fails reports it in status[s] and leaves its x untouched (the null result and the
 * errors[s] entry of SolveBatch); a malformed call (null arrays, count < 0) returns GS_ERR_INVALID_ARG. */
enum gs_ls_status {
    GS_LS_OK = 0,
    GS_LS_SINGULAR = 1,        /* a pivot fell below 1e-12 x max(1, |A(k,k)|), or x is not finite: no result */
    GS_LS_NON_FINITE_INPUT = 2,/* a value is not finite, or the right-hand side is not finite and the matrix is not
                                * singular (the reference's ArgumentException; it factors before it checks b, so a
                                * singular matrix reports GS_LS_SINGULAR whatever its right-hand side) */
    GS_LS_MALFORMED = 3        /* this system's CSR is malformed (offsets, a column out of range or twice) */
};
int gs_sparse_solve_batch(gs_ctx *ctx, int32_t count, const int32_t *n, const int32_t *row_ptr,
                          const int32_t *col_idx, const double *values, const double *rhs, double *x,
                          int32_t *status);

/* The topology verdicts of a set of single-branch outages (host only, no device needed): splits[k] = 1 when
 * removing branch_idx[k] leaves more connected parts than the grid has (ContingencyAnalysis.Splits, :1665);
 * unsolvable[k] = 1 when the grid without it has a part that ProvablyUnsolvablePart (:1750-1830) rejects at
 * `tolerance`. -1 is the intact grid. Bridges and per-side sums come from one depth-first pass, so the cost
 * is O(buses + branches) plus the buses of each slack-less side. Either output may be NULL. */
int gs_outage_topology(const gs_grid_desc *desc, double tolerance, int32_t n_out, const int32_t *branch_idx,
                       uint8_t *splits, uint8_t *unsolvable);

/* ---- uneven multi-grid batch -------------------------------------------------------------------
 * counts[k] independent load flows of grid k (k < n_grids; grids of any sizes, one context) in ONE
 * persistent kernel launch, captured in a CUDA graph: every CTA takes the next (grid, case) item from a
 * device counter, largest grids first, and runs that case's whole Newton iteration itself (mismatch and
 * Jacobian, status test, level-scheduled LU, triangular solves, FP64 refinement in mixed precision, damped
 * update) with no host round trip. The CTA size and the shared-memory use of the level walk are picked by a
 * built-in autotuner on the first call for a set of grids (timed trial launches on a sample of the items),
 * and kept for later calls with the same set.
 * Many SparseNewtonRaphsonPowerFlow.Solve calls (src/GridSim.Core/PowerFlow/SparseNewtonRaphsonPowerFlow.cs:48-54)
 * on different grids, each case from its case's stored voltages.
 * Per-case arrays are concatenated grid after grid, case after case: load_scale (NULL = 1) and the states
 * vm / va_deg (may be NULL) hold counts[k] * n_bus(k) values for grid k; outage, status, iterations and
 * max_mismatch hold one value per case (outage NULL or -1 = none).
 * With Q limits or the DC retry (ContingencyAnalysis.StudyOptions) a case's system changes between Newton passes,
 * which the one-CTA-per-case solve does not carry: each grid's cases then run as one gs_pf_solve_batch, and stats
 * reports the CUDA-event time around them, the cases and the summed iterations (no CTA shape). */
/* ---- schedule of a grid's batched solves, and its autotuner (no counterpart in the reference: GridSim solves one
 *      system at a time) ------------------------------------------------------------------------- */
typedef struct gs_schedule {
    int32_t factor_cut;  /* the factorisation's persistent walk starts at the lowest level from which every level's
                            phases hold at most factor_cut x 16 items; the levels below run one launch each (default 2) */
    int32_t solve_cut;   /* the same cut for the triangular solves (default 2) */
    int32_t tail_max;    /* the few-systems path (one CTA or cluster per system) takes over once at most this many
                            systems still step, 1..296 (default 296) */
    int32_t candidates;  /* out (gs_screen_tune): schedules timed */
    double default_ms;   /* out (gs_screen_tune): device time of the sample's Newton batch under the schedule the grid
                            had before the call */
    double tuned_ms;     /* out (gs_screen_tune): the same under the schedule chosen */
    int32_t subtree_cut; /* the factorisation's unit levels up to this one run as one launch of independent subtrees
                            (one CTA per subtree and system group, level by level with block barriers, so a subtree's
                            entries are re-read from cache); -1 = every level its own launch (default) */
    int32_t reserved[3];
} gs_schedule;

/* The schedule in force on a grid, and setting one (factor_cut, solve_cut >= 1; tail_max clamped to 1..296;
 * subtree_cut >= -1, clamped below the factorisation's persistent walk). */
int gs_grid_schedule_get(gs_grid *g, gs_schedule *out);
int gs_grid_schedule_set(gs_grid *g, const gs_schedule *sched);

/* Autotune the grid's schedule on a sample screen: the outages idx[0 .. n_out) (at most one batch) solved as
 * gs_n1_screen solves them under `opts` (warm start from the base case when set), timed with CUDA events for each
 * candidate (the few-systems threshold of 74, 148 or 296 systems, then the factorisation cut of 1, 2 or 4, then the
 * solve cut of 1, 2 or 4, then the subtree cut: off or the levels whose subtrees hold at most 16, 64 or 256 KB of FP32
 * LU for a system group, each the best of two runs), the fastest kept on the grid for every later solve and screen.
 * `out` gets the schedule chosen and both times. Q limits: the schedule of the grid analysed for them is tuned. */
int gs_screen_tune(gs_grid *g, int32_t n_out, const int32_t *idx, const gs_pf_opts *opts, gs_schedule *out);

typedef struct gs_multi_stats {
    double device_ms;          /* the graph launch (CUDA events) */
    double tune_ms;            /* autotuning trials of this call (0 when the choice was cached) */
    int32_t threads_per_cta;   /* the autotuner's choice */
    int32_t ctas;              /* persistent CTAs launched */
    int32_t items;             /* load flows */
    int32_t tuned_now;         /* 1: this call ran the autotuner */
    int64_t system_steps;      /* Newton steps taken, summed over the cases */
    int32_t shared_top;        /* the autotuner's choice: 1 = the top of the elimination tree in shared memory */
    int32_t reserved[7];
} gs_multi_stats;

int gs_pf_solve_multi(gs_ctx *ctx, int32_t n_grids, gs_grid *const *grids, const int32_t *counts,
                      const double *load_scale, const int32_t *outage, const gs_pf_opts *opts, int32_t *status,
                      int32_t *iterations, double *max_mismatch, double *vm, double *va_deg, gs_multi_stats *stats);

/* ---- request loop (serving) ---------------------------------------------------------------------
 * The reference's nearest counterpart is its sequential `gridsim rpc` host (src/GridSim.Cli/RpcCommand.cs:11-50):
 * one JSON request at a time, `solve` running the `pf` solver on a case held by handle. Here one native
 * scheduler thread keeps every registered grid resident on the device (symbolic data, base solution and a
 * batch of request slots) and steps the occupied slots of each grid one Newton iteration at a time on that
 * grid's own stream (continuous batching): a request joins a free slot of its grid at the next iteration
 * boundary and leaves as soon as its system stops, so requests that arrive while others are on the GPU
 * overlap with them, and grids step concurrently. Slot counts are sized from free device memory when a grid
 * is added (admission by free HBM); a request waits on the host until its grid has a free slot. A system's
 * arithmetic does not depend on its slot or on the other requests: a request's result is the same alone
 * and in any mix. Outage requests start from the grid's solved base case when pf.warm_start_from_base is
 * set; base-case requests (outage -1) start from the case's stored voltages, as gs_pf_solve does.
 * With Q limits or the DC retry (the options of the reference's rpc solve, RpcCommand.cs:675-676) a request's system
 * changes between Newton passes, so it is not stepped in a slot: the loop answers each grid's queued requests with
 * one gs_pf_solve_batch (every request from the case's stored voltages; warm starts are refused with these options),
 * and requests that arrive meanwhile wait for the next batch. That batch runs on the context's stream and the grid's
 * own workspace: while such a loop runs, make no other solve call on its context. */
typedef struct gs_server gs_server;

#define GS_SERVE_MAX_SLOTS 128

typedef struct gs_serve_opts {
    gs_pf_opts pf;             /* options of every request (precision, tolerance, iteration cap, warm start) */
    int32_t slots_per_grid;    /* the most concurrent systems a grid may hold, a multiple of 32, at most
                                  GS_SERVE_MAX_SLOTS; 0 = 128. A grid starts with 32 slots and grows by 32 while its
                                  requests queue and the budget below holds the memory (admission by device memory) */
    int32_t state_slots;       /* solved states returned per grid and iteration; 0 = 16 */
    double hbm_fraction;       /* share of the free device memory (at gs_serve_create) that all grids' slot batches
                                  share; 0 = 0.5 */
    int32_t scheduler_threads; /* host threads that launch the grids' iterations (each owns every k-th grid); 0 = one
                                  per grid up to 8; the batch mode (Q limits, the DC retry, partial pivoting) uses one */
    int32_t reserved[7];
} gs_serve_opts;

typedef struct gs_request {
    int32_t grid;              /* index from gs_serve_add_grid */
    int32_t outage;            /* in-service branch index, -1 = the intact grid */
    int32_t want_state;        /* return the solved Vm and Va */
    int32_t reserved;
    uint64_t tag;              /* the caller's, returned unchanged */
} gs_request;

typedef struct gs_response {
    uint64_t ticket;           /* from gs_serve_submit */
    uint64_t tag;
    int32_t grid, outage;
    int32_t status;            /* enum gs_pf_status */
    int32_t iterations;
    double max_mismatch;       /* pu */
    double queue_ms;           /* submit -> admitted into a slot (host clock) */
    double latency_ms;         /* submit -> result on the host */
    int64_t state_offset;      /* Vm at state[state_offset + i], Va (degrees) at state[state_offset + n_bus + i]; -1 none */
} gs_response;

typedef struct gs_serve_stats {
    int64_t submitted, completed, ticks;  /* ticks: Newton iterations stepped, over all grids */
    int64_t system_steps;                 /* systems stepped, summed over ticks */
    int32_t grids, slots_total, in_flight, queued;
    double slot_bytes;                    /* device memory of the slot batches */
    int32_t failed;                       /* a CUDA error stopped the loop (gs_last_error has it) */
    int32_t reserved[7];
} gs_serve_stats;

int gs_serve_create(gs_ctx *ctx, const gs_serve_opts *opts, gs_server **out);
/* Register a grid (before gs_serve_start): solves its base case when warm starts are on, sizes its slot
 * batch from the memory budget (GS_ERR_OOM when not even 32 slots fit). The grid must outlive the server. */
int gs_serve_add_grid(gs_server *srv, gs_grid *grid, int32_t *grid_index);
int gs_serve_start(gs_server *srv);
/* Queue n requests; tickets[n] (may be NULL) receives their tickets. The whole call is refused
 * (GS_ERR_INVALID_ARG) if any request names an unknown grid or a branch that is not in service. */
int gs_serve_submit(gs_server *srv, int32_t n, const gs_request *req, uint64_t *tickets);
/* Take up to `max` finished requests, waiting up to timeout_ms for the first. States of requests that
 * asked for them are copied into `state` (capacity in doubles); a response whose state does not fit stays
 * queued for the next poll. */
int gs_serve_poll(gs_server *srv, int32_t max, int32_t timeout_ms, gs_response *out, double *state,
                  int64_t state_capacity, int32_t *got);
int gs_serve_stats_get(gs_server *srv, gs_serve_stats *stats);
/* Finish every queued and running request (their responses stay pollable), then stop the loop;
 * GS_ERR_TIMEOUT if that takes longer than timeout_ms (the loop is stopped anyway). */
int gs_serve_stop(gs_server *srv, int32_t timeout_ms);
int gs_serve_destroy(gs_server *srv);

/* ---- allocation-free mismatch check (no counterpart in the reference) ---------------------
 * For callers that must not allocate device memory where they check a state: a host whose device memory is
 * all handed out up front by its own pool (a managed host that reserves its budget once, a process held to a
 * fixed share of a shared GPU), or a latency-bound loop, where cudaMalloc / cudaFree may synchronise the whole
 * device. Computes, for `count` states of the grid, the FP64 max |mismatch| over the grid's equations into
 * d_max_mismatch[count] (NaN for a non-finite mismatch): the mismatch under the grid's own bus types and its
 * base generation and load (voltage-dependent loads at the state's voltage), with at most one branch out per state. It does not model what some solve options
 * change (Q-limit PV-to-PQ switches, load scalings, generator and bus outages, outage sets), so for solves
 * with those it is not the quantity the solver tested. d_vm / d_va are the caller's DEVICE arrays,
 * system-major [count][n_bus], angles in radians; d_outage (device, [count], -1 = none) may be NULL. No
 * device memory is allocated or freed: the only scratch is a file-scope device array sized for
 * GS_NOALLOC_MAX_SYSTEMS systems (16 bytes each: 1 MiB, held by every GPU that loads the library until the
 * process exits). More systems than that are refused with GS_ERR_CAPACITY. The first call on a context
 * looks up that array's device address, so make that first call before any stream capture. Every call
 * shares the array (cleared at the start of each call): calls that overlap on the GPU race, so issue them
 * one after another. Synchronous on the context's stream. */
#define GS_NOALLOC_MAX_SYSTEMS 65536
int gs_pf_mismatch_noalloc(gs_grid *grid, int32_t count, const double *d_vm, const double *d_va,
                           const int32_t *d_outage, double *d_max_mismatch);

#ifdef __cplusplus
}
#endif
#endif /* GRIDSIM_B200_H */
