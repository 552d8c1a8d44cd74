"""Python mirror of GridSim.Core's load-flow seams over the gridsim_b200 C ABI.

* :class:`SparseNewtonRaphsonPowerFlow` — ``IPowerFlowSolver.Solve(GridModel, PowerFlowOptions)``
  (``src/GridSim.Core/Abstractions/IPowerFlowSolver.cs:10-13``) on the B200 engine.
* :class:`ContingencyAnalysis` — ``ScreenBranches`` / ``ScreenBranchesParallel`` / ``ScreenBaseCase`` /
  ``NetAgainstBase`` (``src/GridSim.Core/Analysis/ContingencyAnalysis.cs:306-344, 958-1043``), ``ScreenOutage``
  and the N-k screens (:356-426), ``ScreenElementOutages`` (:1309-1437), with the screen's Newton solves and
  ScreenStateCore classification running on the device.
* :class:`CudaSparseLinearSolver` — ``ISparseLinearSolver`` / ``IBatchedSparseLinearSolver``.
* :class:`UnevenBatch` — many load flows of different grids in one persistent launch.

Every call goes through ``libgridsim_b200.so``; if the library is missing the import of this module
succeeds but the first solve raises (there is no CPU path).
"""
from __future__ import annotations

import ctypes
import itertools
import math
from dataclasses import dataclass, field, replace
from typing import Optional, Sequence

import numpy as np

from . import _abi
from .model import GridModel

# ---------------------------------------------------------------------------------------------


@dataclass
class PowerFlowOptions:
    """PowerFlowOptions (``PowerFlow/PowerFlowOptions.cs``). Q-limit enforcement (PV -> PQ switching passes,
    up to 100, with the reference's reverts) and the DC-angle retry of stalled solves run for single solves, batch
    solves and screens, and through batch solves in the multi-grid batch and the request loop. Both default to off
    here (the reference defaults them on, ``PowerFlowOptions.cs:98,121``) because the benchmark workloads run
    without them. ``flat_start`` reaches the library as the flat-start copy of the model (:meth:`device_model`)."""
    tolerance: float = 1e-8
    max_iterations: int = 30
    diverge_limit_pu: float = 10.0
    flat_start: bool = False
    enforce_q_limits: bool = False
    retry_from_dc_start: bool = False
    per_bus_voltage_limits: bool = False
    precision: str = "fp64"          # "fp64" or "mixed" (FP32 LU and solves, FP64 mismatch and update)
    warm_start_from_base: bool = False
    batch_width: int = 0
    phase_timing: bool = False
    post_fault_rating: str = "A"     # "A", "B" or "C": the rating outage states are judged against (screens)
    max_q_limit_passes: int = 100    # MaxQLimitPasses
    revert_q_limits: bool = False    # RevertQLimits
    # every Newton step by the per-system partial-pivoting LU (the reference's factorisation, FP64) instead of the
    # batched static-pivot factorisation; that LU runs anyway for a system whose static pivot collapses
    partial_pivoting: bool = False

    def to_c(self) -> _abi.PfOpts:
        o = _abi.default_opts()
        o.tolerance = float(self.tolerance)
        o.max_iterations = int(self.max_iterations)
        o.diverge_limit_pu = float(self.diverge_limit_pu)
        o.flat_start = int(self.flat_start)
        o.enforce_q_limits = int(self.enforce_q_limits)
        o.retry_from_dc_start = int(self.retry_from_dc_start)
        o.per_bus_voltage_limits = int(self.per_bus_voltage_limits)
        o.precision = {"fp64": _abi.PREC_FP64, "mixed": _abi.PREC_MIXED}[self.precision]
        o.warm_start_from_base = int(self.warm_start_from_base)
        o.batch_width = int(self.batch_width)
        o.phase_timing = int(self.phase_timing)
        o.post_fault_rating = {"A": _abi.RATE_A, "B": _abi.RATE_B, "C": _abi.RATE_C}[self.post_fault_rating.upper()]
        o.max_q_limit_passes = int(self.max_q_limit_passes)
        o.revert_q_limits = int(self.revert_q_limits)
        o.partial_pivoting = int(self.partial_pivoting)
        return o

    def device_model(self, model: GridModel) -> GridModel:
        """The model whose descriptor the library solves with these options: the flat-start copy under
        ``flat_start`` (the library takes a flat start through the descriptor's voltages), else `model`."""
        return model.flat_started() if self.flat_start else model

    def device_c(self) -> _abi.PfOpts:
        """gs_pf_opts for a grid built from :meth:`device_model`: the flat start is already in its voltages."""
        return replace(self, flat_start=False).to_c()


# ContingencyAnalysis.StudyOptions (ContingencyAnalysis.cs:263-268): 100 iterations with Q limits on.
STUDY_MAX_ITERATIONS = 100


def study_options(precision: str = "fp64") -> "PowerFlowOptions":
    """ContingencyAnalysis.StudyOptions: the options every contingency study of the reference solves with (100
    iterations, Q limits on, and the reference's default DC-angle retry, ``PowerFlowOptions.cs:121``)."""
    return PowerFlowOptions(max_iterations=STUDY_MAX_ITERATIONS, enforce_q_limits=True, retry_from_dc_start=True,
                            precision=precision)


@dataclass
class LineFlow:
    loading_percent: float
    sf_mva: complex
    st_mva: complex


@dataclass
class PowerFlowResult:
    """PowerFlowResult (``PowerFlow/PowerFlowResult.cs``)."""
    status: int
    iterations: int
    max_mismatch: float
    bus_ids: np.ndarray
    vm: np.ndarray
    va_deg: np.ndarray
    p_inj_mw: np.ndarray
    q_inj_mvar: np.ndarray
    loading_percent: np.ndarray
    sf_mva: np.ndarray
    st_mva: np.ndarray

    @property
    def converged(self) -> bool:
        return self.status == _abi.PF_CONVERGED

    @property
    def status_name(self) -> str:
        return _abi.PF_STATUS_NAMES[self.status]

    @property
    def total_loss_mw(self) -> float:
        return float(np.sum(self.p_inj_mw))


class EngineError(RuntimeError):
    pass


# ---------------------------------------------------------------------------------------------
class CudaContext:
    """An open device (gs_ctx): bounded probe and FP64 self-test on creation."""

    _default: Optional["CudaContext"] = None

    def __init__(self, device: int = 0, probe_timeout_ms: int = 10000):
        self.lib = _abi.load_library()
        self.handle = ctypes.c_void_p()
        o = _abi.CtxOpts()
        o.probe_timeout_ms = probe_timeout_ms
        rc = self.lib.gs_ctx_create(device, ctypes.byref(o), ctypes.byref(self.handle))
        if rc != _abi.GS_OK:
            raise EngineError(f"gs_ctx_create({device}) failed: {self.lib.gs_status_str(rc).decode()}")

    @classmethod
    def default(cls) -> "CudaContext":
        if cls._default is None:
            cls._default = CudaContext(0)
        return cls._default

    def last_error(self) -> str:
        buf = ctypes.create_string_buffer(1024)
        self.lib.gs_last_error(self.handle, buf, 1024)
        return buf.value.decode()

    def check(self, rc: int, what: str) -> None:
        if rc != _abi.GS_OK:
            raise EngineError(f"{what}: {self.lib.gs_status_str(rc).decode()}: {self.last_error()}")

    def close(self) -> None:
        if self.handle:
            self.lib.gs_ctx_destroy(self.handle)
            self.handle = ctypes.c_void_p()


class CudaGrid:
    """A grid uploaded with its shared symbolic analysis (gs_grid)."""

    def __init__(self, model: GridModel, ctx: Optional[CudaContext] = None):
        self.ctx = ctx or CudaContext.default()
        self.model = model
        self.handle = ctypes.c_void_p()
        d = model.desc()
        self.ctx.check(self.ctx.lib.gs_grid_create(self.ctx.handle, ctypes.byref(d), ctypes.byref(self.handle)),
                       "gs_grid_create")

    def info(self) -> _abi.GridInfo:
        i = _abi.GridInfo()
        self.ctx.check(self.ctx.lib.gs_grid_info_get(self.handle, ctypes.byref(i)), "gs_grid_info_get")
        return i

    def schedule(self) -> dict:
        """The batched-solve schedule in force (gs_grid_schedule_get): factor_cut, solve_cut, tail_max, subtree_cut."""
        sc = _abi.Schedule()
        self.ctx.check(self.ctx.lib.gs_grid_schedule_get(self.handle, ctypes.byref(sc)), "gs_grid_schedule_get")
        return {"factor_cut": sc.factor_cut, "solve_cut": sc.solve_cut, "tail_max": sc.tail_max,
                "subtree_cut": sc.subtree_cut}

    def set_schedule(self, factor_cut: int = 2, solve_cut: int = 2, tail_max: int = 296, subtree_cut: int = -1) -> None:
        """gs_grid_schedule_set; the defaults are the schedule a grid starts with."""
        sc = _abi.Schedule()
        sc.factor_cut, sc.solve_cut, sc.tail_max = int(factor_cut), int(solve_cut), int(tail_max)
        sc.subtree_cut = int(subtree_cut)
        self.ctx.check(self.ctx.lib.gs_grid_schedule_set(self.handle, ctypes.byref(sc)), "gs_grid_schedule_set")

    def close(self) -> None:
        if self.handle:
            self.ctx.lib.gs_grid_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------------------------
class SparseNewtonRaphsonPowerFlow:
    """IPowerFlowSolver on the B200 engine. One instance per thread (as the reference's engines)."""

    def __init__(self, precision: str = "fp64", ctx: Optional[CudaContext] = None):
        self.precision = precision
        self.ctx = ctx
        self._grid: Optional[CudaGrid] = None
        self._model_key = None
        self._flat_src: Optional[GridModel] = None
        self._flat: Optional[GridModel] = None

    def grid_for(self, model: GridModel, options: Optional[PowerFlowOptions] = None) -> CudaGrid:
        """The device grid of `model` (kept while the same model is solved again); with options that ask for a flat
        start, the grid of its flat-start copy (:meth:`PowerFlowOptions.device_model`), kept likewise."""
        if options is not None and options.flat_start:
            if self._flat_src is not model:
                self._flat_src, self._flat = model, options.device_model(model)
            model = self._flat
        key = id(model)
        if self._grid is None or self._model_key != key or self._grid.model is not model:
            self._grid = CudaGrid(model, self.ctx)
            self._model_key = key
        return self._grid

    def solve(self, model: GridModel, options: Optional[PowerFlowOptions] = None) -> PowerFlowResult:
        opt = options or PowerFlowOptions(precision=self.precision)
        g = self.grid_for(model, opt)
        n, nb = model.n_bus, model.n_branch
        out = {k: np.zeros(n) for k in ("vm", "va_deg", "p_inj_mw", "q_inj_mvar")}
        out["loading_percent"] = np.zeros(nb)
        out["sf"] = np.zeros(2 * max(nb, 1))
        out["st"] = np.zeros(2 * max(nb, 1))
        r = _abi.PfResult()
        r.vm, r.va_deg, r.p_inj_mw, r.q_inj_mvar = (_p(out[k]) for k in ("vm", "va_deg", "p_inj_mw", "q_inj_mvar"))
        r.loading_pct, r.sf_mva, r.st_mva = _p(out["loading_percent"]), _p(out["sf"]), _p(out["st"])
        c = opt.device_c()
        g.ctx.check(g.ctx.lib.gs_pf_solve(g.handle, ctypes.byref(c), ctypes.byref(r)), "gs_pf_solve")
        sf = out["sf"][: 2 * nb].reshape(-1, 2)
        st = out["st"][: 2 * nb].reshape(-1, 2)
        return PowerFlowResult(status=r.status, iterations=r.iterations, max_mismatch=r.max_mismatch,
                               bus_ids=model.bus_id.copy(), vm=out["vm"], va_deg=out["va_deg"],
                               p_inj_mw=out["p_inj_mw"], q_inj_mvar=out["q_inj_mvar"],
                               loading_percent=out["loading_percent"], sf_mva=sf[:, 0] + 1j * sf[:, 1],
                               st_mva=st[:, 0] + 1j * st[:, 1])

    def solve_batch(self, model: GridModel, load_scale: Optional[np.ndarray] = None,
                    outage: Optional[np.ndarray] = None, options: Optional[PowerFlowOptions] = None,
                    keep_states: bool = False) -> dict:
        """Many load flows of one grid in device batches (``gs_pf_solve_batch``)."""
        opt = options or PowerFlowOptions(precision=self.precision)
        g = self.grid_for(model, opt)
        n = model.n_bus
        count = (load_scale.shape[0] if load_scale is not None else outage.shape[0])
        ls = None if load_scale is None else np.ascontiguousarray(load_scale, np.float64)
        og = None if outage is None else np.ascontiguousarray(outage, np.int32)
        st = np.zeros(count, np.int32)
        it = np.zeros(count, np.int32)
        mis = np.zeros(count)
        vm = np.zeros(count * n) if keep_states else None
        va = np.zeros(count * n) if keep_states else None
        c = opt.device_c()
        g.ctx.check(g.ctx.lib.gs_pf_solve_batch(g.handle, count, _p(ls), _p(og), ctypes.byref(c), _p(st), _p(it),
                                                _p(mis), _p(vm), _p(va)), "gs_pf_solve_batch")
        out = {"status": st, "iterations": it, "max_mismatch": mis}
        if keep_states:
            out["vm"] = vm.reshape(count, n)
            out["va_deg"] = va.reshape(count, n)
        return out


# ---------------------------------------------------------------------------------------------
class CudaSparseLinearSolver:
    """ISparseLinearSolver (``Abstractions/ISparseLinearSolver.cs:12-17``) and IBatchedSparseLinearSolver
    (``Abstractions/IBatchedSparseLinearSolver.cs:19-37``) on the device: ``gs_sparse_solve_batch``.

    A matrix is a SciPy CSR matrix or a tuple ``(indptr, indices, data)`` of a square n x n matrix. ``solve`` returns
    x, or None when the matrix is singular, and raises ValueError on non-finite input or a malformed matrix (the
    reference's ArgumentException). ``solve_batch`` takes systems of any sizes and patterns; a failed system's entry is
    None and its exception goes into ``errors``; the inputs are never modified."""

    def __init__(self, ctx: Optional[CudaContext] = None):
        self.ctx = ctx or CudaContext.default()

    @staticmethod
    def _csr(a):
        if hasattr(a, "indptr"):
            return (np.asarray(a.indptr), np.asarray(a.indices), np.asarray(a.data), a.shape[0])
        indptr, indices, data = a
        return (np.asarray(indptr), np.asarray(indices), np.asarray(data), len(indptr) - 1)

    def solve(self, a, b) -> Optional[np.ndarray]:
        errors = [None]
        (x,) = self.solve_batch([a], [b], errors)
        if errors[0] is not None:
            raise errors[0]
        return x

    def solve_batch(self, matrices: Sequence, rhs: Sequence, errors: Optional[list] = None) -> list:
        if len(matrices) != len(rhs):
            raise ValueError(f"{len(matrices)} matrices but {len(rhs)} right-hand sides")
        k = len(matrices)
        if errors is not None and len(errors) != k:
            raise ValueError("errors must hold one slot per system")
        parts = [self._csr(a) for a in matrices]
        for (indptr, _, _, n), b in zip(parts, rhs):
            if len(indptr) != n + 1 or np.asarray(b).shape != (n,):
                raise ValueError("a matrix is not square or its right-hand side has the wrong length")
        n = np.array([p[3] for p in parts], np.int32)
        rp = np.concatenate([np.asarray(p[0], np.int32) for p in parts]) if k else np.zeros(0, np.int32)
        ci = np.concatenate([np.asarray(p[1], np.int32) for p in parts]) if k else np.zeros(0, np.int32)
        va = np.concatenate([np.asarray(p[2], np.float64) for p in parts]) if k else np.zeros(0)
        bb = np.concatenate([np.asarray(b, np.float64) for b in rhs]) if k else np.zeros(0)
        x = np.zeros(bb.shape[0])
        st = np.zeros(k, np.int32)
        rc = self.ctx.lib.gs_sparse_solve_batch(self.ctx.handle, k, _p(n), _p(rp), _p(ci), _p(va), _p(bb), _p(x), _p(st))
        self.ctx.check(rc, "gs_sparse_solve_batch")
        out, off = [], 0
        for j in range(k):
            nj = int(n[j])
            err = None
            if st[j] == _abi.LS_OK:
                out.append(x[off:off + nj].copy())
            else:
                out.append(None)
                if st[j] == _abi.LS_NON_FINITE_INPUT:
                    err = ValueError(f"system {j}: a value or right-hand side is not finite")
                elif st[j] == _abi.LS_MALFORMED:
                    err = ValueError(f"system {j}: the CSR matrix is malformed")
            if errors is not None:
                errors[j] = err
            off += nj
        return out


class UnevenBatch:
    """Independent load flows of several grids of any sizes in one persistent launch (``gs_pf_solve_multi``).

    The grids are uploaded once; every :meth:`solve` runs ``counts[k]`` cases of grid k, each from its case's
    stored voltages, optionally with per-bus load multipliers and a branch outage. The CTA shape is autotuned on
    the first call for this set of grids and reused afterwards. With Q limits or the DC retry (StudyOptions) each
    grid's cases run as one batch solve instead."""

    def __init__(self, models: Sequence[GridModel], ctx: Optional[CudaContext] = None):
        self.ctx = ctx or CudaContext.default()
        self.models = list(models)
        self.grids = [CudaGrid(m, self.ctx) for m in self.models]
        self._flat_grids: Optional[list] = None
        self.stats = None

    def solve(self, counts: Sequence[int], load_scale: Optional[Sequence[np.ndarray]] = None,
              outage: Optional[Sequence[np.ndarray]] = None, options: Optional[PowerFlowOptions] = None,
              keep_states: bool = False) -> dict:
        """load_scale[k]: [counts[k], n_bus(k)] multipliers of Pd and Qd; outage[k]: [counts[k]] branch indices.
        Returns per-grid lists of status, iterations, max_mismatch (and vm, va_deg [counts[k], n_bus(k)])."""
        opt = options or PowerFlowOptions()
        counts = np.ascontiguousarray(counts, np.int32)
        k = len(self.models)
        n = [m.n_bus for m in self.models]
        total = int(counts.sum())
        states = int(sum(int(c) * nb for c, nb in zip(counts, n)))
        ls = None if load_scale is None else np.ascontiguousarray(
            np.concatenate([np.asarray(load_scale[g], np.float64).reshape(-1) for g in range(k)]))
        og = None if outage is None else np.ascontiguousarray(
            np.concatenate([np.asarray(outage[g], np.int32).reshape(-1) for g in range(k)]))
        if ls is not None and ls.shape[0] != states:
            raise ValueError("load_scale: counts[k] x n_bus(k) values per grid")
        if og is not None and og.shape[0] != total:
            raise ValueError("outage: counts[k] values per grid")
        st, it, mis = np.zeros(total, np.int32), np.zeros(total, np.int32), np.zeros(total)
        vm = np.zeros(states) if keep_states else None
        va = np.zeros(states) if keep_states else None
        grids = self.grids
        if opt.flat_start:   # the flat-start copies, uploaded on first use
            if self._flat_grids is None:
                self._flat_grids = [CudaGrid(opt.device_model(m), self.ctx) for m in self.models]
            grids = self._flat_grids
        handles = (ctypes.c_void_p * max(k, 1))(*[g.handle.value for g in grids])
        c = opt.device_c()
        stats = _abi.MultiStats()
        self.ctx.check(self.ctx.lib.gs_pf_solve_multi(self.ctx.handle, k, handles, _p(counts), _p(ls), _p(og),
                                                      ctypes.byref(c), _p(st), _p(it), _p(mis), _p(vm), _p(va),
                                                      ctypes.byref(stats)), "gs_pf_solve_multi")
        self.stats = {f: getattr(stats, f) for f, _ in _abi.MultiStats._fields_ if f != "reserved"}
        out = {"status": [], "iterations": [], "max_mismatch": [], "vm": [], "va_deg": []}
        c0 = s0 = 0
        for g in range(k):
            cnt = int(counts[g])
            out["status"].append(st[c0:c0 + cnt])
            out["iterations"].append(it[c0:c0 + cnt])
            out["max_mismatch"].append(mis[c0:c0 + cnt])
            if keep_states:
                out["vm"].append(vm[s0:s0 + cnt * n[g]].reshape(cnt, n[g]))
                out["va_deg"].append(va[s0:s0 + cnt * n[g]].reshape(cnt, n[g]))
            c0 += cnt
            s0 += cnt * n[g]
        return out

    def close(self) -> None:
        for g in self.grids + (self._flat_grids or []):
            g.close()
        self.grids = []
        self._flat_grids = None


# ---------------------------------------------------------------------------------------------
@dataclass
class ContingencyViolation:
    """ContingencyViolation (ContingencyAnalysis.cs:156-163)."""
    kind: int      # _abi.VIOL_*
    element: int   # original branch index, or bus id
    value: float   # loading % or Vm pu
    name: str = ""


@dataclass
class ContingencyResult:
    """ContingencyResult (ContingencyAnalysis.cs:9-96)."""
    outage: str
    converged: bool
    max_branch_loading_percent: float
    worst_boundary_loading_percent: float
    min_vm: float
    max_vm: float
    violations: list
    details: list = field(default_factory=list)
    status: int = _abi.PF_CONVERGED
    iterations: int = 0
    max_mismatch: float = 0.0
    netted_against_base: bool = False
    pre_existing_violations: list = field(default_factory=list)
    worsened_pre_existing_violations: list = field(default_factory=list)
    islanded: bool = False  # not converged, and the outage split the network (:1661-1665)
    kind: int = 0           # OutageKind: 0 branch, 1 generator, 2 bus
    lost_load_mw: float = 0.0
    lost_generation_mw: float = 0.0
    note: Optional[str] = None

    @property
    def secure(self) -> bool:
        return self.converged and len(self.violations) == 0


def _branch_label(model: GridModel, k: int) -> str:
    """ContingencyAnalysis.Label (:1832-1833): the name (else "from-to" bus ids) plus " (tx)"."""
    nm = model.br_name[k] if model.br_name is not None else ""
    lab = nm if nm else f"{int(model.bus_id[model.br_from[k]])}-{int(model.bus_id[model.br_to[k]])}"
    return lab + (" (tx)" if model.is_transformer[k] else "")


def _violation_texts(model: GridModel, details: Sequence[ContingencyViolation]) -> list:
    """ContingencyAnalysis.ViolationTexts (:1050-1067): branch and boundary lines in detail order, then one
    undervoltage and one overvoltage line."""
    texts = []
    for d in details:
        if d.kind == _abi.VIOL_BRANCH_OVERLOAD:
            texts.append(f"branch {d.name} {d.value:.0f}%")
        elif d.kind == _abi.VIOL_BOUNDARY_OVERLOAD:
            texts.append(f"boundary {d.name} {d.value:.0f}%")
    under = [d.value for d in details if d.kind == _abi.VIOL_UNDERVOLTAGE]
    over = [d.value for d in details if d.kind == _abi.VIOL_OVERVOLTAGE]
    if under:
        texts.append(f"undervoltage {min(under):.3f} p.u.")
    if over:
        texts.append(f"overvoltage {max(over):.3f} p.u.")
    return texts


def _branch_name(model: GridModel, k: int) -> str:
    """The name a branch violation carries: the branch's name, else "from-to" (:1168-1172)."""
    return model.branch_label(k)


# ---- shared outage dispatch (OutageDispatch.GovernorDroop / Inertia) ---------------------------------------
# ConverterPlant.Types (Model/Model.cs:207-215): plant types that are converter-interfaced ('_' read as '-')
CONVERTER_TYPES = frozenset({"wind", "onshore", "offshore", "wind-onshore", "wind-offshore", "solar", "pv", "storage",
                             "battery", "bess", "interconnector", "hvdc", "tidal"})


def _synchronous(model: GridModel) -> np.ndarray:
    """Per unit: a synchronous machine with a governor, neither power-flow-only nor converter plant
    (Generator.IsConverterInterfaced, Model/Model.cs:147: the flag, else the type)."""
    mc = model.machines()
    out = np.zeros(model.n_gen, bool)
    for g in range(model.n_gen):
        conv = (bool(mc["converter"][g]) if mc["converter"][g] >= 0
                else (mc["gen_type"][g] or "").strip().lower().replace("_", "-") in CONVERTER_TYPES)
        out[g] = not mc["pf_only"][g] and not conv
    return out


def participation_weights(model: GridModel, units: Sequence[int], bus_type: np.ndarray, dispatch: str,
                          island: Optional[Sequence[int]] = None, removed_bus: int = -1) -> np.ndarray:
    """ParticipationWeights (ContingencyAnalysis.cs:1588-1645) over the network after an outage: `units` are the
    units left (model positions, model order), `bus_type` the bus types after it, `removed_bus` a bus gone with its
    branches (-1: none), `island` bus positions of the part that lost the power (None: everywhere). A unit takes
    part when it is synchronous and its bus reaches a reference bus over in-service branches (inside that part);
    its weight is its machine base (MBase, or the system base when MBase is 0 or less, MachineBase.EffectiveMva)
    for droop and H times that for inertia. ValueError for a participant whose Pmin is above its Pmax."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    n = model.n_bus
    on = (model.br_in_service != 0) & (model.br_from != removed_bus) & (model.br_to != removed_bus)
    f, t = model.br_from[on], model.br_to[on]
    graph = coo_matrix((np.ones(f.shape[0]), (f, t)), shape=(n, n))
    _, part = connected_components(graph, directed=False)

    def flood(seeds):   # the buses in-service branches connect to a seed: the seeds' connected parts
        return np.isin(part, part[np.asarray(seeds, np.int64)]) if len(seeds) else np.zeros(n, bool)

    reach = flood([i for i in range(n) if bus_type[i] == 3 and i != removed_bus])
    if island is not None:
        reach &= flood([int(i) for i in island])
    mc = model.machines()
    sync = _synchronous(model)
    how = "governor droop" if dispatch == "droop" else "inertia"
    w = np.zeros(len(units))
    for p, g in enumerate(units):
        if not sync[g] or not reach[int(model.gen_bus[g])]:
            continue
        mva = float(mc["mbase"][g]) if mc["mbase"][g] > 0.0 else float(model.base_mva)
        x = mva if dispatch == "droop" else float(mc["inertia_h"][g]) * mva
        if not (x > 0.0) or not math.isfinite(x):
            continue
        if mc["pmin"][g] > mc["pmax"][g]:
            raise ValueError(f"Outage sharing by {how}: generator {p} at bus {int(model.bus_id[model.gen_bus[g]])} "
                             f"has Pmin {mc['pmin'][g]:g} MW above Pmax {mc['pmax'][g]:g} MW, so it has no dispatch "
                             "range to share within.")
        w[p] = x
    return w


def share_lost_power(model: GridModel, units: Sequence[int], bus_type: np.ndarray, lost_mw: float, dispatch: str,
                     island: Optional[Sequence[int]] = None, removed_bus: int = -1):
    """ShareLostPower (ContingencyAnalysis.cs:1509-1579): the net lost MW (positive: generation lost) shared among
    the participants of :func:`participation_weights` in proportion to their weights, each within [Pmin, Pmax]
    from its scheduled output; a unit whose share exceeds its headroom is fixed at its limit and the rest shared
    again among the others, until every share fits or no unit is left (what is left goes to the reference bus).
    Returns (the new scheduled output of each unit of `units`, the note)."""
    if dispatch not in ("droop", "inertia"):
        raise ValueError("ShareLostPower shares among units; the reference-bus mode does not share.")
    if not math.isfinite(lost_mw):
        raise ValueError("The lost power must be a finite number of MW.")
    how = "governor droop" if dispatch == "droop" else "inertia"
    pg = np.array([float(model.pg[g]) for g in units])
    if lost_mw == 0.0:
        return pg, f"no net power lost, nothing to share by {how}"
    weights = participation_weights(model, units, bus_type, dispatch, island, removed_bus)
    mc = model.machines()
    raise_ = lost_mw > 0.0
    weight, room, delta, active = {}, {}, np.zeros(len(units)), []
    for p, g in enumerate(units):
        if not (weights[p] > 0.0):
            continue
        r = float(mc["pmax"][g]) - pg[p] if raise_ else pg[p] - float(mc["pmin"][g])
        if not (r > 0.0):
            continue
        weight[p], room[p] = float(weights[p]), r
        active.append(p)
    remaining = abs(lost_mw)
    at_limit = 0
    participants = len(active)
    while active and remaining > 0.0:
        wsum = 0.0
        for p in active:
            wsum += weight[p]
        capped = [p for p in active if remaining * weight[p] / wsum > room[p]]
        if not capped:
            for p in active:
                delta[p] += remaining * weight[p] / wsum
            remaining = 0.0
            break
        for p in capped:
            delta[p] += room[p]
            remaining -= room[p]
            active.remove(p)
            at_limit += 1
        if remaining < 0.0:
            remaining = 0.0
    sign = 1.0 if raise_ else -1.0
    for p in range(len(units)):
        if delta[p] != 0.0:
            pg[p] = pg[p] + sign * delta[p]
    note = f"{'lost' if raise_ else 'surplus'} {abs(lost_mw):.1f} MW shared by {how} over {participants} unit(s)"
    if at_limit > 0:
        note += f", {at_limit} at a limit"
    if remaining > 0.0:
        note += f"; {remaining:.1f} MW beyond their headroom left to the reference"
    return pg, note


def _shared_outage(model: GridModel, kind: int, index: int, dispatch: str):
    """The shared dispatch of one element outage, as ScreenElementOutage builds it (:1355-1421): None when nothing
    is shared (a branch outage, or no unit left to take the reference); else (the model to solve the outage on, or
    None when no power was lost, and the sharing note). The model keeps every element, so the device removes the
    unit or bus as usual; its remaining units carry the shared output and its reference is already re-elected."""
    if kind == 0:
        return None
    on = [int(g) for g in np.nonzero(model.gen_in_service)[0]]
    types = model.bus_type.copy()
    if kind == 1:
        bus = int(model.gen_bus[index])
        new_ref, moved_note = ContingencyAnalysis._reelect(model, index, -1, bus)
        if new_ref is None and moved_note is not None:   # no unit left to take the reference: nothing is solved
            return None
        units = [g for g in on if g != index]
        lost, island, removed = float(model.pg[index]), [bus], -1
        affected = bus
    else:
        new_ref, moved_note = ContingencyAnalysis._reelect(model, -1, index, index)
        if new_ref is None and moved_note is not None:
            return None
        units = [g for g in on if int(model.gen_bus[g]) != index]
        lost_gen = 0.0
        for g in on:
            if int(model.gen_bus[g]) == index:
                lost_gen += float(model.pg[g])
        lost = lost_gen - float(model.pd[index])
        touch = (model.br_in_service != 0) & ((model.br_from == index) | (model.br_to == index))
        other = np.where(model.br_from[touch] == index, model.br_to[touch], model.br_from[touch])
        island = [int(x) for x in other if x != index]
        removed = affected = index
    if new_ref is not None:   # ReelectReference: the old reference (or the removed bus) PQ, the new one a reference
        types[affected] = 1
        types[new_ref] = 3
    pg, note = share_lost_power(model, units, types, lost, dispatch, island, removed)
    if lost == 0.0:
        return None, note
    moved = model.copy()
    moved.bus_type = types
    moved.pg[units] = pg
    return moved, note


def _merge_rows(raw: dict, subs: dict, keep_states: bool) -> None:
    """Replace rows of a screen's raw result with single-outage results ({row: raw of one outage})."""
    for key in ("status", "iterations", "max_mismatch", "min_vm", "max_vm", "max_loading_pct", "worst_boundary_pct",
                "islanded"):
        for j, s in subs.items():
            raw[key][j] = s[key][0]
    if keep_states:
        for j, s in subs.items():
            raw["vm"][j] = s["vm"][0]
            raw["va_deg"][j] = s["va_deg"][0]
    ptr = raw["viol_ptr"]
    rows = []
    for j in range(ptr.shape[0] - 1):
        src, a, b = (subs[j], 0, subs[j]["viol_ptr"][1]) if j in subs else (raw, ptr[j], ptr[j + 1])
        rows.append((src["viol_kind"][a:b], src["viol_element"][a:b], src["viol_value"][a:b]))
    raw["viol_ptr"] = np.concatenate([[0], np.cumsum([len(r[0]) for r in rows])]).astype(np.int32)
    for q, key in enumerate(("viol_kind", "viol_element", "viol_value")):
        raw[key] = (np.concatenate([r[q] for r in rows]) if rows else raw[key][:0]).astype(raw[key].dtype)


@dataclass
class NkScreenReport:
    """NkScreenReport (``ContingencyAnalysis.cs:174-186``): the screened combinations worst first, the single
    outages left out of the pairing because they already fail at N-1, and why nothing was screened (or None)."""
    results: list
    excluded_single_outages: list
    note: Optional[str] = None


class ContingencyAnalysis:
    """The N-1 branch screen of ``Analysis/ContingencyAnalysis.cs`` on the B200 engine."""

    WORSENED_LOADING_MARGIN_PERCENT = 1.0   # :986
    WORSENED_VOLTAGE_MARGIN_PU = 0.005      # :990
    BASE_CASE_LABEL = "base case"           # :279

    @staticmethod
    def screen_raw(model: GridModel, branch_indices: Sequence[int], solver: SparseNewtonRaphsonPowerFlow,
                   options: PowerFlowOptions, keep_states: bool = False) -> dict:
        """One ``gs_n1_screen`` call; returns the raw arrays (status, iterations, violation CSR, ...)."""
        idx = np.ascontiguousarray(branch_indices, dtype=np.int32)
        return ContingencyAnalysis._screen_call(model, idx, None, solver, options, keep_states)

    @staticmethod
    def tune_screen(model: GridModel, branch_indices: Sequence[int], solver: SparseNewtonRaphsonPowerFlow,
                    options: PowerFlowOptions) -> dict:
        """``gs_screen_tune``: time the candidate schedules (few-systems threshold, factorisation and solve cuts) on
        the Newton batch of these outages under `options` and keep the fastest on the solver's grid for its later
        screens. Returns the schedule chosen, the candidates timed and the sample's device time before and after."""
        g = solver.grid_for(model, options)
        idx = np.ascontiguousarray(branch_indices, dtype=np.int32)
        sc = _abi.Schedule()
        c = options.device_c()
        g.ctx.check(g.ctx.lib.gs_screen_tune(g.handle, idx.shape[0], _p(idx), ctypes.byref(c), ctypes.byref(sc)),
                    "gs_screen_tune")
        return {"factor_cut": sc.factor_cut, "solve_cut": sc.solve_cut, "tail_max": sc.tail_max,
                "subtree_cut": sc.subtree_cut, "candidates": sc.candidates, "default_ms": sc.default_ms,
                "tuned_ms": sc.tuned_ms}

    @staticmethod
    def screen_sets_raw(model: GridModel, branch_sets, solver: SparseNewtonRaphsonPowerFlow,
                        options: PowerFlowOptions, keep_states: bool = False) -> dict:
        """One ``gs_nk_screen`` call: row j of `branch_sets` ([n_out, k], -1 = none) lists the branches outage j
        takes out together (ScreenOutageCore over several indices, ``ContingencyAnalysis.cs:1087-1097``)."""
        sets = np.ascontiguousarray(branch_sets, dtype=np.int32)
        if sets.ndim != 2:
            raise ValueError("branch_sets must be [n_out, k]")
        return ContingencyAnalysis._screen_call(model, sets, sets.shape[1], solver, options, keep_states)

    @staticmethod
    def screen_elements_raw(model: GridModel, kinds: Sequence[int], indices: Sequence[int],
                            solver: SparseNewtonRaphsonPowerFlow, options: PowerFlowOptions,
                            keep_states: bool = False, dispatch: str = "reference") -> dict:
        """``gs_element_screen``: outage j is the branch / generator / bus indices[j] of kinds[j] (0, 1, 2);
        generator indices are positions in the model's generator arrays, bus indices bus positions.

        `dispatch` is OutageDispatch (ContingencyAnalysis.cs:120-129): "reference" (the reference bus picks up the
        lost power; one device call for every outage), "droop" or "inertia" (ShareLostPower moves the remaining
        units' scheduled output first, :1370-1374 and :1410-1421). A shared outage is solved as the element outage
        of its own grid: the model with the units moved and the reference already re-elected (ReelectReference
        works on the output before the sharing), so each costs a grid upload; "share_notes" holds the sharing notes
        (None where nothing was shared: branch outages, and outages that leave no unit to take the reference)."""
        if dispatch not in ("reference", "droop", "inertia"):
            raise ValueError(f"unknown outage dispatch {dispatch!r}: reference, droop or inertia")
        if dispatch != "reference" and options.warm_start_from_base:
            raise ValueError("a shared outage dispatch solves each outage from the model's stored voltages, as the "
                             "reference does; warm_start_from_base is not offered with it")
        k = np.ascontiguousarray(kinds, dtype=np.int32)
        idx = np.ascontiguousarray(indices, dtype=np.int32)
        raw = ContingencyAnalysis._screen_call(model, idx, ("elements", k), solver, options, keep_states)
        if dispatch == "reference":
            return raw
        notes = [None] * k.shape[0]
        own = SparseNewtonRaphsonPowerFlow(solver.precision, solver.ctx)
        subs = {}
        for j in range(k.shape[0]):
            plan = _shared_outage(model, int(k[j]), int(idx[j]), dispatch)
            if plan is None:
                continue
            moved, notes[j] = plan
            if moved is None:  # nothing to share: the reference-bus solve is the state
                continue
            subs[j] = ContingencyAnalysis._screen_call(moved, idx[j:j + 1], ("elements", k[j:j + 1]), own, options,
                                                       keep_states)
            if own._grid is not None:
                own._grid.close()
                own._grid = None
        raw["share_notes"] = notes
        if subs:
            _merge_rows(raw, subs, keep_states)
        return raw

    @staticmethod
    def _screen_call(model, idx, width, solver, options, keep_states):
        g = solver.grid_for(model, options)
        k = idx.shape[0]
        n = model.n_bus
        # violation capacity: remembered per grid (a too small buffer makes the engine report the size
        # needed, and the screen is run again)
        cap = max(256, 16 * k, int(getattr(g, "viol_per_outage", 0) * k * 1.25) + 64)
        while True:
            out = dict(status=np.zeros(k, np.int32), iterations=np.zeros(k, np.int32), max_mismatch=np.zeros(k),
                       min_vm=np.zeros(k), max_vm=np.zeros(k), max_loading_pct=np.zeros(k),
                       worst_boundary_pct=np.zeros(k), islanded=np.zeros(k, np.uint8),
                       viol_ptr=np.zeros(k + 1, np.int32), viol_kind=np.zeros(cap, np.int32),
                       viol_element=np.zeros(cap, np.int32), viol_value=np.zeros(cap))
            if keep_states:
                out["vm"] = np.zeros(k * n)
                out["va_deg"] = np.zeros(k * n)
            r = _abi.N1Result()
            for key, v in out.items():
                setattr(r, key, _p(v))
            r.viol_capacity = cap
            c = options.device_c()
            if width is None:
                rc = g.ctx.lib.gs_n1_screen(g.handle, k, _p(idx), ctypes.byref(c), ctypes.byref(r))
            elif isinstance(width, tuple):
                rc = g.ctx.lib.gs_element_screen(g.handle, k, _p(width[1]), _p(idx), ctypes.byref(c), ctypes.byref(r))
            else:
                rc = g.ctx.lib.gs_nk_screen(g.handle, k, width, _p(idx), ctypes.byref(c), ctypes.byref(r))
            if rc == _abi.GS_ERR_CAPACITY:
                cap = r.viol_count + 64
                g.viol_per_outage = max(getattr(g, "viol_per_outage", 0), r.viol_count / max(k, 1))
                continue
            g.ctx.check(rc, "gs_n1_screen" if width is None else
                        "gs_element_screen" if isinstance(width, tuple) else "gs_nk_screen")
            break
        nv = r.viol_count
        for key in ("viol_kind", "viol_element", "viol_value"):
            out[key] = out[key][:nv]
        if keep_states:
            out["vm"] = out["vm"].reshape(k, n)
            out["va_deg"] = out["va_deg"].reshape(k, n)
        out.update(base_status=r.base_status, base_iterations=r.base_iterations, device_ms=r.device_ms,
                   n_singular_pivot=r.n_singular_pivot, n_partial_pivot=r.n_partial_pivot, n_batches=r.n_batches, kernel_launches=r.kernel_launches,
                   newton_iterations=r.newton_iterations, factor_ms=r.factor_ms, solve_ms=r.solve_ms,
                   mismatch_ms=r.mismatch_ms, other_ms=r.other_ms, factor_bytes=r.factor_bytes,
                   level_factor_ms=r.level_factor_ms, level_factor_bytes=r.level_factor_bytes, tail_ms=r.tail_ms)
        return out

    @staticmethod
    def outage_topology(model: GridModel, branch_indices: Sequence[int], tolerance: float = 1e-8):
        """Per outage (-1 = the intact grid): (splits, unsolvable) — ContingencyAnalysis.Splits (:1665) and whether
        ProvablyUnsolvablePart (:1750-1830) rejects the grid without the branch. Host only (no device needed); the
        screen runs the same pass before it solves."""
        lib = _abi.load_library()
        idx = np.ascontiguousarray(branch_indices, dtype=np.int32)
        sp = np.zeros(idx.shape[0], np.uint8)
        un = np.zeros(idx.shape[0], np.uint8)
        d = model.desc()
        rc = lib.gs_outage_topology(ctypes.byref(d), float(tolerance), idx.shape[0], _p(idx), _p(sp), _p(un))
        if rc != _abi.GS_OK:
            raise EngineError(f"gs_outage_topology: {_abi.load_library().gs_status_str(rc).decode()}")
        return sp.astype(bool), un.astype(bool)

    @classmethod
    def _results(cls, model: GridModel, idx, raw: dict, labels: Optional[Sequence[str]] = None) -> list:
        """ContingencyResult per outage; `idx` holds a branch per outage (-1 = the intact grid) or, for the
        multi-branch screen, a row of branches (-1 = none) labelled "A + B" (LabelMany, :1836-1837); `labels`
        replaces those labels."""
        res = []
        for j, k in enumerate(idx):
            st = int(raw["status"][j])
            br = [int(x) for x in np.atleast_1d(k) if x >= 0]
            label = " + ".join(_branch_label(model, b) for b in br) if br else cls.BASE_CASE_LABEL
            if labels is not None:
                label = labels[j]
            if st != _abi.PF_CONVERGED:  # NonConverged (:1661-1662)
                isl = bool(raw["islanded"][j])
                res.append(ContingencyResult(label, False, 0.0, 0.0, 0.0, 0.0, ["islanded" if isl else "no solution"],
                                             [], st, int(raw["iterations"][j]), float(raw["max_mismatch"][j]),
                                             islanded=isl))
                continue
            a, b = raw["viol_ptr"][j], raw["viol_ptr"][j + 1]
            det = []
            for q in range(a, b):
                kind = int(raw["viol_kind"][q])
                el = int(raw["viol_element"][q])
                name = (_branch_name(model, el) if kind == _abi.VIOL_BRANCH_OVERLOAD
                        else model.boundaries[el][0] if kind == _abi.VIOL_BOUNDARY_OVERLOAD else "")
                det.append(ContingencyViolation(kind, el, float(raw["viol_value"][q]), name))
            res.append(ContingencyResult(label, True, float(raw["max_loading_pct"][j]),
                                         float(raw["worst_boundary_pct"][j]), float(raw["min_vm"][j]),
                                         float(raw["max_vm"][j]), _violation_texts(model, det), det, st,
                                         int(raw["iterations"][j]), float(raw["max_mismatch"][j])))
        return res

    @classmethod
    def screen_branches(cls, model: GridModel, solver: Optional[SparseNewtonRaphsonPowerFlow] = None,
                        options: Optional[PowerFlowOptions] = None,
                        branch_indices: Optional[Sequence[int]] = None) -> list:
        """ScreenBranches / ScreenBranchesParallel / ScreenBranchesBatched: results in branch order."""
        solver = solver or SparseNewtonRaphsonPowerFlow()
        options = options or PowerFlowOptions(precision=solver.precision)
        idx = model.in_service_branches() if branch_indices is None else np.asarray(branch_indices, np.int32)
        raw = cls.screen_raw(model, idx, solver, options)
        return cls._results(model, idx, raw)

    screen_branches_parallel = screen_branches
    screen_branches_batched = screen_branches

    @classmethod
    def screen_base_case(cls, model: GridModel, solver: Optional[SparseNewtonRaphsonPowerFlow] = None,
                         options: Optional[PowerFlowOptions] = None) -> ContingencyResult:
        """ScreenBaseCase (:958-962): the intact grid through the same classification."""
        solver = solver or SparseNewtonRaphsonPowerFlow()
        options = options or PowerFlowOptions(precision=solver.precision)
        raw = cls.screen_raw(model, np.array([-1], np.int32), solver, options)
        return cls._results(model, [-1], raw)[0]

    @classmethod
    def screen_outage(cls, model: GridModel, indices: Sequence[int],
                      solver: Optional[SparseNewtonRaphsonPowerFlow] = None,
                      options: Optional[PowerFlowOptions] = None) -> ContingencyResult:
        """ScreenOutage (:1087-1097 via ScreenOutageCore): the given branches out together, solved and classified."""
        solver = solver or SparseNewtonRaphsonPowerFlow()
        options = options or PowerFlowOptions(precision=solver.precision)
        row = np.array([list(indices) or [-1]], np.int32)
        raw = cls.screen_sets_raw(model, row, solver, options)
        return cls._results(model, row, raw)[0]

    STRESS_VOLTAGE_WEIGHT_PER_PU = 1000.0   # :239
    DEFAULT_CANDIDATE_COUNT = 20            # :245
    MAX_COMBINATIONS = 20_000_000           # ANA-18

    @classmethod
    def stress_score(cls, c: ContingencyResult) -> float:
        """StressScore (:1077-1084): branch plus boundary loading plus 1000 x the voltage excursion beyond the
        0.94-1.06 band; a state that did not converge is +inf."""
        if not c.converged:
            return math.inf
        s = c.max_branch_loading_percent + c.worst_boundary_loading_percent
        s += max(0.0, 0.94 - c.min_vm) * cls.STRESS_VOLTAGE_WEIGHT_PER_PU
        s += max(0.0, c.max_vm - 1.06) * cls.STRESS_VOLTAGE_WEIGHT_PER_PU
        return s

    @classmethod
    def screen_n_minus_k_report(cls, model: GridModel, k: int, solver: Optional[SparseNewtonRaphsonPowerFlow] = None,
                                options: Optional[PowerFlowOptions] = None, candidate_count: int = 20,
                                exhaustive: bool = False) -> "NkScreenReport":
        """ScreenNMinusKReport (:378-426): the N-1 screen first (unless exhaustive), the single outages that solve
        ranked by stress_score (stable, ties in branch order) and the top max(candidate_count, k) kept (RankCandidates
        :438-451), every k-subset of the candidates in lexicographic order (Combinations :1851-1866) screened on the
        device in one call, results worst first (stable)."""
        solver = solver or SparseNewtonRaphsonPowerFlow()
        options = options or PowerFlowOptions(precision=solver.precision)
        return cls._nk_report(model, k, lambda idx: cls.screen_raw(model, idx, solver, options),
                              lambda sets: cls.screen_sets_raw(model, sets, solver, options), candidate_count,
                              exhaustive)

    @classmethod
    def _nk_report(cls, model: GridModel, k: int, screen_single, screen_sets, candidate_count: int,
                   exhaustive: bool) -> "NkScreenReport":
        """The N-k pipeline over two raw screens (a branch list, and a [n_out, k] set array)."""
        if k < 1:
            raise ValueError("contingency depth k must be >= 1")
        live = model.in_service_branches()
        n = live.shape[0]
        if k > n:
            return NkScreenReport([], [], f"the model has {n} branch(es), fewer than the depth k = {k}, so no "
                                          f"{k}-outage combination exists; nothing was screened.")
        if k == 1:
            return NkScreenReport(cls._results(model, live, screen_single(live)), [])
        excluded = []
        if exhaustive:
            cand = live
        else:
            single = cls._results(model, live, screen_single(live))
            solvable = [i for i, c in enumerate(single) if c.converged]
            excluded = [c for c in single if not c.converged]
            take = min(max(candidate_count, k), len(solvable))
            ranked = sorted(solvable, key=lambda i: -cls.stress_score(single[i]))[:take]
            cand = live[np.array(ranked, dtype=np.int64)] if ranked else live[:0]
        count = math.comb(len(cand), k) if len(cand) >= k else 0
        if count > cls.MAX_COMBINATIONS:
            raise ValueError(f"N-{k}: {len(cand)} candidate branches give about {count:.4g} outage combinations, "
                             f"more than the {cls.MAX_COMBINATIONS} one screen takes; screen fewer candidates (a "
                             f"candidate count) or a smaller k.")
        note = None
        if len(cand) < k:
            note = (f"only {len(cand)} single outage(s) solve ({len(excluded)} do not), fewer than the depth k = {k}, "
                    f"so no {k}-outage combination could be formed; nothing was screened.")
            return NkScreenReport([], excluded, note)
        combos = np.array(list(itertools.combinations([int(c) for c in cand], k)), np.int32).reshape(-1, k)
        results = cls._results(model, combos, screen_sets(combos))
        order = sorted(range(len(results)), key=lambda i: -cls.stress_score(results[i]))
        return NkScreenReport([results[i] for i in order], excluded, note)

    @classmethod
    def screen_n_minus_k(cls, model: GridModel, k: int, solver: Optional[SparseNewtonRaphsonPowerFlow] = None,
                         options: Optional[PowerFlowOptions] = None, candidate_count: int = 20,
                         exhaustive: bool = False) -> list:
        """ScreenNMinusK (:370-373): the results of screen_n_minus_k_report."""
        return cls.screen_n_minus_k_report(model, k, solver, options, candidate_count, exhaustive).results

    @classmethod
    def screen_n_minus_2(cls, model: GridModel, solver: Optional[SparseNewtonRaphsonPowerFlow] = None,
                         options: Optional[PowerFlowOptions] = None, candidate_count: int = 20,
                         exhaustive: bool = False) -> list:
        """ScreenNMinus2 (:356-360)."""
        return cls.screen_n_minus_k(model, 2, solver, options, candidate_count, exhaustive)

    @staticmethod
    def single_outages(model: GridModel, branches: bool = True, generators: bool = False,
                       buses: bool = False) -> list:
        """SingleOutages (:1294-1302): (kind, index) for every branch (branch order), then every in-service generator
        (model order; the index is its position among the in-service units, as GridModel.Generators), then every
        bus (model order)."""
        out = []
        if branches:
            out += [(0, k) for k in range(model.n_branch)]
        if generators:
            out += [(1, k) for k in range(int(np.sum(model.gen_in_service != 0)))]
        if buses:
            out += [(2, i) for i in range(model.n_bus)]
        return out

    @staticmethod
    def _reelect(model: GridModel, removed_gen: int, removed_bus: int, affected: int):
        """ReelectReference (:1440-1488) for the note: (new reference bus position or None, note text or None)."""
        if model.bus_type[affected] != 3:
            return None, None
        on = np.nonzero(model.gen_in_service)[0]
        units = [g for g in on if g != removed_gen and int(model.gen_bus[g]) != removed_bus]
        if removed_bus < 0 and any(int(model.gen_bus[g]) == affected for g in units):
            return None, None
        adj = [[] for _ in range(model.n_bus)]
        for k in np.nonzero(model.br_in_service)[0]:
            f, t = int(model.br_from[k]), int(model.br_to[k])
            if removed_bus in (f, t):
                continue
            adj[f].append(t)
            adj[t].append(f)
        if removed_bus < 0:
            seeds = [affected]
        else:
            seeds = [int(model.br_to[k]) if int(model.br_from[k]) == removed_bus else int(model.br_from[k])
                     for k in np.nonzero(model.br_in_service)[0] if removed_bus in (int(model.br_from[k]), int(model.br_to[k]))]
        reach, queue = set(seeds), list(seeds)
        while queue:
            u = queue.pop(0)
            for v in adj[u]:
                if v != removed_bus and v not in reach:
                    reach.add(v)
                    queue.append(v)
        best = None
        for g in units:
            if int(model.gen_bus[g]) in reach and (best is None or abs(model.pg[g]) > abs(model.pg[best])):
                best = g
        aid = int(model.bus_id[affected])
        if best is None:
            return None, f"no in-service unit is left to take over the reference of bus {aid}"
        return int(model.gen_bus[best]), f"reference moved from bus {aid} to bus {int(model.bus_id[model.gen_bus[best]])}"

    @classmethod
    def screen_element_outages(cls, model: GridModel, outages: Sequence, solver: Optional[SparseNewtonRaphsonPowerFlow] = None,
                               options: Optional[PowerFlowOptions] = None, dispatch: str = "reference") -> list:
        """ScreenElementOutages (:1309-1320): every (kind, index) of `outages` (SingleOutages' indexing), results in
        order with the reference's labels ("gen 3 at bus 7", "bus 7"), lost load and generation and the notes (the
        reference move, then the sharing). `dispatch`: "reference" (one device call for every outage), "droop" or
        "inertia" (:meth:`screen_elements_raw`)."""
        solver = solver or SparseNewtonRaphsonPowerFlow()
        options = options or PowerFlowOptions(precision=solver.precision)
        on = np.nonzero(model.gen_in_service)[0]
        kinds = np.array([int(k) for k, _ in outages], np.int32)
        idx = np.array([int(on[i]) if k == 1 else int(i) for k, i in outages], np.int32)
        raw = cls.screen_elements_raw(model, kinds, idx, solver, options, dispatch=dispatch)
        labels = []
        for j, (k, i) in enumerate(outages):
            if k == 0:
                labels.append(_branch_label(model, int(idx[j])))
            elif k == 1:  # "gen {index} at bus {id}" for a unit without a name (:1363)
                labels.append(f"gen {i} at bus {int(model.bus_id[model.gen_bus[idx[j]]])}")
            else:
                labels.append(f"bus {int(model.bus_id[i])}")
        res = cls._results(model, np.where(kinds == 0, idx, -1), raw, labels)
        for j, (k, i) in enumerate(outages):
            r = res[j]
            r.kind = int(k)
            if k == 1:
                g = int(idx[j])
                r.lost_generation_mw = float(model.pg[g])
                r.note = cls._reelect(model, g, -1, int(model.gen_bus[g]))[1]
            elif k == 2:
                r.lost_load_mw = float(model.pd[i])
                r.lost_generation_mw = float(sum(model.pg[g] for g in on if int(model.gen_bus[g]) == i))
                r.note = cls._reelect(model, -1, int(i), int(i))[1]
            shared = raw.get("share_notes", [None] * len(res))[j]
            if shared is not None:
                r.note = shared if r.note is None else r.note + "; " + shared
        return res

    @classmethod
    def net_against_base(cls, model: GridModel, outage: ContingencyResult, base: ContingencyResult,
                         count_worsened: bool = False) -> ContingencyResult:
        """NetAgainstBase (:1000-1034)."""
        if not base.converged:
            raise ValueError("Contingency netting: the base case did not converge, so there is no base state to net "
                             "the outage violations against.")
        import dataclasses
        if not outage.converged:
            return dataclasses.replace(outage, netted_against_base=True)
        before = {(v.kind, v.element): v.value for v in base.details}
        fresh, pre, worse = [], [], []
        for v in outage.details:
            if (v.kind, v.element) not in before:
                fresh.append(v)
                continue
            b = before[(v.kind, v.element)]
            if v.kind == _abi.VIOL_UNDERVOLTAGE:
                w = v.value < b - cls.WORSENED_VOLTAGE_MARGIN_PU
            elif v.kind == _abi.VIOL_OVERVOLTAGE:
                w = v.value > b + cls.WORSENED_VOLTAGE_MARGIN_PU
            else:
                w = v.value > b + cls.WORSENED_LOADING_MARGIN_PERCENT
            if w:
                worse.append(v)
            (fresh if (w and count_worsened) else pre).append(v)
        return dataclasses.replace(outage, violations=_violation_texts(model, fresh),
                                   pre_existing_violations=_violation_texts(model, pre),
                                   worsened_pre_existing_violations=_violation_texts(model, worse),
                                   netted_against_base=True)
