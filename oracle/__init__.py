"""CPU ORACLE for the gridsim_b200 load-flow path — TEST INFRASTRUCTURE ONLY.

Python binding of ``oracle/gs_oracle.cpp``, the C++17 restatement of GridSim.Core's FP64 sparse
Gilbert-Peierls Newton-Raphson load flow and N-1 screen. Only the tests, the smoke check and the
benchmark's CPU-baseline leg may import this package, and only as the checker; the engine never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from gridsim_b200 import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "gs_oracle.cpp")
_LIB = os.path.join(_HERE, "_build", "libgs_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with g++ (the recipe is this function: one source file, no dependencies)."""
    os.makedirs(os.path.dirname(_LIB), exist_ok=True)
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        subprocess.check_call(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", "-o", _LIB, _SRC])
    return _LIB


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(_LIB)
        vp, i32 = ctypes.c_void_p, ctypes.c_int32
        lib.gso_pf_solve.argtypes = [ctypes.POINTER(_abi.GridDesc), ctypes.POINTER(_abi.PfOpts),
                                     ctypes.POINTER(_abi.PfResult)]
        lib.gso_n1_screen.argtypes = [ctypes.POINTER(_abi.GridDesc), i32, vp, ctypes.POINTER(_abi.PfOpts), i32,
                                      ctypes.POINTER(_abi.N1Result)]
        lib.gso_jacobian.argtypes = [ctypes.POINTER(_abi.GridDesc), vp, vp, vp, vp, vp, i32, vp, i32]
        lib.gso_md_order.argtypes = [i32, vp, vp, vp]
        lib.gso_nk_screen.argtypes = [ctypes.POINTER(_abi.GridDesc), i32, i32, vp, ctypes.POINTER(_abi.PfOpts), i32,
                                      ctypes.POINTER(_abi.N1Result)]
        lib.gso_element_screen.argtypes = [ctypes.POINTER(_abi.GridDesc), i32, vp, vp, ctypes.POINTER(_abi.PfOpts), i32,
                                           ctypes.POINTER(_Machines), vp, ctypes.POINTER(_abi.N1Result)]
        lib.gso_share_lost_power.argtypes = [ctypes.POINTER(_abi.GridDesc), ctypes.c_double, ctypes.POINTER(_Machines),
                                             i32, vp, vp, vp]
        lib.gso_outage_topology.argtypes = [ctypes.POINTER(_abi.GridDesc), ctypes.c_double, i32, vp, vp, vp]
        lib.gso_sparse_solve.argtypes = [i32, vp, vp, vp, vp, vp]
        lib.gso_ilu0_apply.argtypes = [i32, vp, vp, vp, vp, vp]
        lib.gso_bicgstab.argtypes = [i32, vp, vp, vp, vp, ctypes.c_double, i32, vp]
        lib.gso_max_mismatch.argtypes = [ctypes.POINTER(_abi.GridDesc), i32, vp, vp, vp, vp]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class _Machines(ctypes.Structure):
    _fields_ = [("dispatch", ctypes.c_int32), ("pmin", ctypes.c_void_p), ("pmax", ctypes.c_void_p),
                ("mbase", ctypes.c_void_p), ("h", ctypes.c_void_p), ("sync", ctypes.c_void_p)]


DISPATCH = {"reference": 0, "droop": 1, "inertia": 2}

# ConverterPlant.Types (Model/Model.cs:207-215): converter-interfaced plant by type, case-insensitive, '_' as '-'
CONVERTER_TYPES = {"wind", "onshore", "offshore", "wind-onshore", "wind-offshore", "solar", "pv", "storage", "battery",
                   "bess", "interconnector", "hvdc", "tidal"}


def _machines(model, dispatch):
    """Per descriptor unit: Pmin, Pmax, MBase, H and whether it is a synchronous machine with a governor (not
    power-flow-only; converter flag, else inferred from the type, Generator.IsConverterInterfaced :147)."""
    mc = model.machines()
    conv = [bool(c) if c >= 0 else (t or "").strip().lower().replace("_", "-") in CONVERTER_TYPES
            for c, t in zip(mc["converter"], mc["gen_type"])]
    sync = np.array([0 if (pf or cv) else 1 for pf, cv in zip(mc["pf_only"], conv)], np.uint8)
    keep = [np.ascontiguousarray(mc[k], np.float64) for k in ("pmin", "pmax", "mbase", "inertia_h")] + [sync]
    s = _Machines(DISPATCH[dispatch], *[_p(a) for a in keep])
    return s, keep


def share_note(stats, dispatch) -> str:
    """The note ShareLostPower writes (ContingencyAnalysis.cs:1515-1578) from its figures (lost MW, participants,
    units at a limit, MW left to the reference)."""
    how = "governor droop" if dispatch == "droop" else "inertia"
    lost, parts, at_limit, left = float(stats[0]), int(stats[1]), int(stats[2]), float(stats[3])
    if lost == 0.0:
        return f"no net power lost, nothing to share by {how}"
    note = f"{'lost' if lost > 0 else 'surplus'} {abs(lost):.1f} MW shared by {how} over {parts} unit(s)"
    if at_limit > 0:
        note += f", {at_limit} at a limit"
    if left > 0.0:
        note += f"; {left:.1f} MW beyond their headroom left to the reference"
    return note


def share_lost_power(model, lost_mw, dispatch, island_buses=None):
    """ShareLostPower on `model` itself: (every descriptor unit's Pg after the sharing, the note). `island_buses`:
    bus positions of the part that lost the power (None: the whole network). ValueError where the reference throws."""
    lib = _load()
    mach, keep = _machines(model, dispatch)
    isl = np.ascontiguousarray([] if island_buses is None else island_buses, np.int32)
    pg = np.zeros(model.n_gen)
    stats = np.zeros(4)
    d = model.desc()
    rc = lib.gso_share_lost_power(ctypes.byref(d), float(lost_mw), ctypes.byref(mach),
                                  -1 if island_buses is None else isl.shape[0], _p(isl), _p(pg), _p(stats))
    if rc != 0:
        raise ValueError(f"ShareLostPower refused: lost {lost_mw} MW, dispatch {dispatch}")
    return pg, share_note(stats, dispatch)


def solve(model, opts=None) -> dict:
    """IPowerFlowSolver.Solve with the reference's CPU sparse Newton engine."""
    lib = _load()
    o = opts or _abi.default_opts()
    n, nb = model.n_bus, model.n_branch
    out = {k: np.zeros(n) for k in ("vm", "va_deg", "p_inj_mw", "q_inj_mvar")}
    out["loading_pct"] = np.zeros(nb)
    out["sf_mva"] = np.zeros(2 * nb)
    out["st_mva"] = np.zeros(2 * nb)
    r = _abi.PfResult()
    for k, v in out.items():
        setattr(r, k, _p(v))
    d = model.desc()
    rc = lib.gso_pf_solve(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r))
    if rc != 0:
        raise RuntimeError(f"oracle solve failed: {rc}")
    out.update(status=r.status, iterations=r.iterations, max_mismatch=r.max_mismatch)
    return out


def screen(model, branch_idx, opts=None, threads: int = 0, keep_states: bool = False) -> dict:
    """ScreenBranchesParallel on `threads` host threads (0 = all)."""
    return _screen(model, np.ascontiguousarray(branch_idx, dtype=np.int32), None, opts, threads, keep_states)


def screen_sets(model, sets, opts=None, threads: int = 0, keep_states: bool = False) -> dict:
    """ScreenOutageCore over several branches per outage: `sets` is [n_out, k] (-1 = none)."""
    sets = np.ascontiguousarray(sets, dtype=np.int32)
    return _screen(model, sets, sets.shape[1], opts, threads, keep_states)


def screen_elements(model, kinds, indices, opts=None, threads: int = 0, keep_states: bool = False,
                    dispatch: str = "reference") -> dict:
    """ScreenElementOutages: outage j is the branch / generator / bus indices[j] of kinds[j] (0, 1, 2), its lost
    power picked up by the reference bus, or shared by governor droop or inertia (`dispatch`); with a shared
    dispatch "share" holds each outage's (lost MW, participants, units at a limit, MW left), lost MW NaN where
    nothing was shared, and "notes" the sharing notes (None there)."""
    k = np.ascontiguousarray(kinds, dtype=np.int32)
    return _screen(model, np.ascontiguousarray(indices, dtype=np.int32), ("elements", k, dispatch), opts, threads,
                   keep_states)


def _screen(model, idx, width, opts, threads, keep_states):
    lib = _load()
    o = opts or _abi.default_opts()
    k = idx.shape[0]
    n = model.n_bus
    cap = max(64, k * 8)
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
        d = model.desc()
        if width is None:
            rc = lib.gso_n1_screen(ctypes.byref(d), k, _p(idx), ctypes.byref(o), threads, ctypes.byref(r))
        elif isinstance(width, tuple):
            mach, keep = _machines(model, width[2])
            share = np.zeros(4 * k)
            rc = lib.gso_element_screen(ctypes.byref(d), k, _p(width[1]), _p(idx), ctypes.byref(o), threads,
                                        ctypes.byref(mach), _p(share), ctypes.byref(r))
            out["share"] = share.reshape(k, 4)
        else:
            rc = lib.gso_nk_screen(ctypes.byref(d), k, width, _p(idx), ctypes.byref(o), threads, ctypes.byref(r))
        if rc == _abi.GS_ERR_CAPACITY:
            cap = r.viol_count + 16
            continue
        if rc != 0:
            raise RuntimeError(f"oracle screen failed: {rc}")
        break
    nv = r.viol_count
    for key in ("viol_kind", "viol_element", "viol_value"):
        out[key] = out[key][:nv]
    if keep_states:
        out["vm"] = out["vm"].reshape(k, n)
        out["va_deg"] = out["va_deg"].reshape(k, n)
    out["base_status"] = r.base_status
    out["base_iterations"] = r.base_iterations
    if "share" in out:
        out["notes"] = [None if np.isnan(s[0]) else share_note(s, width[2]) for s in out["share"]]
    return out


def outage_topology(model, branch_idx, tolerance=1e-8):
    """Per outage: (splits, unsolvable) — ContingencyAnalysis.Splits and ProvablyUnsolvablePart of the grid
    without the branch, computed per reduced model as the reference does."""
    lib = _load()
    idx = np.ascontiguousarray(branch_idx, dtype=np.int32)
    sp = np.zeros(idx.shape[0], np.uint8)
    un = np.zeros(idx.shape[0], np.uint8)
    d = model.desc()
    rc = lib.gso_outage_topology(ctypes.byref(d), tolerance, idx.shape[0], _p(idx), _p(sp), _p(un))
    if rc != 0:
        raise RuntimeError(f"oracle topology failed: {rc}")
    return sp.astype(bool), un.astype(bool)


def jacobian(model):
    """The reference's Jacobian (CSR) and mismatch at the model's start point."""
    lib = _load()
    d = model.desc()
    m = ctypes.c_int32()
    nnz = ctypes.c_int32()
    lib.gso_jacobian(ctypes.byref(d), ctypes.byref(m), ctypes.byref(nnz), None, None, None, 0, None, 0)
    rp = np.zeros(m.value + 1, np.int32)
    ci = np.zeros(nnz.value, np.int32)
    val = np.zeros(nnz.value)
    mis = np.zeros(m.value)
    rc = lib.gso_jacobian(ctypes.byref(d), ctypes.byref(m), ctypes.byref(nnz), _p(rp), _p(ci), _p(val), nnz.value,
                          _p(mis), m.value)
    if rc != 0:
        raise RuntimeError(f"oracle jacobian failed: {rc}")
    return rp, ci, val, mis


def max_mismatch(model, vm, va_rad, outage=None):
    """Max |mismatch| of given states ([count][n], angles in radians), each with branch outage[s] out (None: none)."""
    lib = _load()
    vm = np.ascontiguousarray(vm, np.float64)
    va = np.ascontiguousarray(va_rad, np.float64)
    count = vm.shape[0]
    out = np.zeros(count)
    o = None if outage is None else np.ascontiguousarray(outage, np.int32)
    d = model.desc()
    rc = lib.gso_max_mismatch(ctypes.byref(d), count, None if o is None else _p(o), _p(vm), _p(va), _p(out))
    if rc != 0:
        raise RuntimeError(f"oracle mismatch failed: {rc}")
    return out


def md_order(row_ptr, col_idx):
    lib = _load()
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    n = rp.shape[0] - 1
    q = np.zeros(n, np.int32)
    lib.gso_md_order(n, _p(rp), _p(ci), _p(q))
    return q


def sparse_solve(row_ptr, col_idx, val, b):
    """CpuSparseLuSolver.Solve (PowerFlow/CpuSparseLuSolver.cs:30-48): x, or None when the matrix is singular;
    ValueError (the reference's ArgumentException) when it factorises but b has a non-finite entry."""
    lib = _load()
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    v = np.ascontiguousarray(val, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    x = np.zeros(rp.shape[0] - 1)
    rc = lib.gso_sparse_solve(rp.shape[0] - 1, _p(rp), _p(ci), _p(v), _p(bb), _p(x))
    if rc == 2:
        raise ValueError("Sparse LU: the right-hand side has a non-finite entry")
    return None if rc else x


def _csr(row_ptr, col_idx, val):
    return (np.ascontiguousarray(row_ptr, np.int32), np.ascontiguousarray(col_idx, np.int32),
            np.ascontiguousarray(val, np.float64))


def ilu0_apply(row_ptr, col_idx, val, r):
    """Ilu0.Factor(A).Apply(r) (Numerics/Sparse.cs:240-300): z with the ILU(0) factors and the row-relative guard."""
    lib = _load()
    rp, ci, v = _csr(row_ptr, col_idx, val)
    rr = np.ascontiguousarray(r, np.float64)
    z = np.zeros(rp.shape[0] - 1)
    lib.gso_ilu0_apply(rp.shape[0] - 1, _p(rp), _p(ci), _p(v), _p(rr), _p(z))
    return z


def bicgstab(row_ptr, col_idx, val, b, tol=1e-10, max_iter=0):
    """BiCgStab.Solve with the ILU(0) preconditioner (Numerics/Sparse.cs:319-405; tol default
    NumericTolerances.DefaultKrylovTolerance, max_iter 0 = 4n + 200): (accepted, x)."""
    lib = _load()
    rp, ci, v = _csr(row_ptr, col_idx, val)
    bb = np.ascontiguousarray(b, np.float64)
    x = np.zeros(rp.shape[0] - 1)
    rc = lib.gso_bicgstab(rp.shape[0] - 1, _p(rp), _p(ci), _p(v), _p(bb), float(tol), int(max_iter), _p(x))
    return rc == 0, x
