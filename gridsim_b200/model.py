"""Grid model and the two case formats the load-flow path reads.

``GridModel`` holds the fields of GridSim's ``GridModel`` that the load flow uses (Bus
``src/GridSim.Core/Model/Model.cs:20-35``, Generator ``:91-114``, Branch ``:253-275``) as flat numpy
arrays, in model order. Bus references inside the arrays are 0-based positions; ``bus_id`` keeps the
external ids (the key of voltage violations).

Loaders:

* :func:`load_matpower` — MATPOWER ``.m`` files, following ``IO/Matpower/MatpowerParser.cs:128-401``:
  isolated (type 4) buses and out-of-service branches are dropped with everything incident to them,
  out-of-service generators are kept but not solved, a PV bus with no in-service generator is solved
  as PQ, VMAX/VMIN become the bus's own limits, TAP 0 means a line (ratio 1).
* :func:`load_case_dir` / :func:`save_case_dir` — GridSim's v1 JSON case directory
  (``IO/Json/JsonGridLoader.cs:55-255``): ``system.json``, ``buses.json``, ``generation.json``,
  ``demand.json``, ``transmission.json``, ``transformer.json``, ``boundaries.json``. Only the keys this path needs are read; ``"dispatch": false``
  keeps the written generator outputs (``:254``), which is what every case written here uses.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import re
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

PQ, PV, SLACK = 1, 2, 3


# ZipLoad.VariesWithVoltage (Model/Model.cs:49): a load other than pure constant power
def zip_varies(c) -> bool:
    return bool(c[0] != 0 or c[1] != 0 or c[3] != 0 or c[4] != 0)


ZIP_SUM_TOLERANCE = 1e-9  # JsonGridLoader.ZipSumTolerance (IO/Json/JsonGridLoader.cs:385)


def _json_zip(buses) -> Optional[np.ndarray]:
    """The buses' optional "zip" blocks (JsonGridLoader.ParseZip / ParseZipValues, IO/Json/JsonGridLoader.cs:395-427):
    all six coefficients present and finite, each triple summing to 1 within 1e-9, else ValueError naming the bus;
    None when no bus gives one."""
    if not any(b.get("zip") is not None for b in buses):
        return None
    out = np.tile(np.array([0.0, 0.0, 1.0, 0.0, 0.0, 1.0]), (len(buses), 1))
    for i, b in enumerate(buses):
        z = b.get("zip")
        if z is None:
            continue
        where = f"buses.json: bus {b['id']}" + (f" ('{b['name']}')" if b.get("name") is not None else "")
        vals = []
        for key in ("ap", "bp", "cp", "aq", "bq", "cq"):
            v = z.get(key)
            if v is None:
                raise ValueError(f"{where}: zip is missing coefficient '{key}' (all of ap, bp, cp, aq, bq, cq are required).")
            v = float(v)
            if not math.isfinite(v):
                raise ValueError(f"{where}: zip coefficient '{key}' is {v!r}, which is not a finite number.")
            vals.append(v)
        if not abs(sum(vals[:3]) - 1.0) <= ZIP_SUM_TOLERANCE:
            raise ValueError(f"{where}: zip real-power coefficients ap + bp + cp sum to {sum(vals[:3])!r}, not 1.")
        if not abs(sum(vals[3:]) - 1.0) <= ZIP_SUM_TOLERANCE:
            raise ValueError(f"{where}: zip reactive-power coefficients aq + bq + cq sum to {sum(vals[3:])!r}, not 1.")
        out[i] = vals
    return out


@dataclass
class GridModel:
    name: str
    base_mva: float
    # buses
    bus_id: np.ndarray
    bus_type: np.ndarray
    pd: np.ndarray
    qd: np.ndarray
    gs: np.ndarray
    bs: np.ndarray
    vm: np.ndarray
    va_deg: np.ndarray
    vmin: np.ndarray  # NaN = no own limit
    vmax: np.ndarray
    base_kv: np.ndarray
    # generators
    gen_bus: np.ndarray  # bus positions
    pg: np.ndarray
    qg: np.ndarray
    vg: np.ndarray
    qmin: np.ndarray
    qmax: np.ndarray
    gen_in_service: np.ndarray
    # branches
    br_from: np.ndarray  # bus positions
    br_to: np.ndarray
    r: np.ndarray
    x: np.ndarray
    b: np.ndarray
    tap: np.ndarray
    shift_deg: np.ndarray
    rate_a: np.ndarray
    br_in_service: np.ndarray
    is_transformer: np.ndarray
    rate_b: Optional[np.ndarray] = None  # short-term / emergency MVA (0 = not given); None = all 0
    rate_c: Optional[np.ndarray] = None
    br_name: Optional[List[str]] = None  # branch names ("" = unnamed); None = every branch unnamed
    # transmission boundaries (Boundary, Model/Model.cs:516-560): (name, limit MW, [(branch name, direction)])
    boundaries: List[Tuple[str, float, List[Tuple[str, int]]]] = field(default_factory=list)
    # machine data of the units (Generator, Model/Model.cs:91-114), read only by the outage dispatch by governor
    # droop or inertia: Pmin / Pmax (MW), MBase (MVA; 0 or less = the system base), H (s), the plant type, the
    # power-flow-only flag and the converter flag (-1 = inferred from the type). None = the record's defaults.
    pmin: Optional[np.ndarray] = None
    pmax: Optional[np.ndarray] = None
    mbase: Optional[np.ndarray] = None
    inertia_h: Optional[np.ndarray] = None
    gen_type: Optional[List[str]] = None
    pf_only: Optional[np.ndarray] = None
    converter: Optional[np.ndarray] = None
    # voltage-dependent (ZIP) loads (Bus.Zip, Model/Model.cs:33,45-90): [n_bus, 6] Ap Bp Cp Aq Bq Cq, the load drawn at
    # V pu being Pd (Ap V^2 + Bp V + Cp), Qd (Aq V^2 + Bq V + Cq); None = every load constant power (0, 0, 1)
    zip: Optional[np.ndarray] = None
    meta: dict = field(default_factory=dict)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_bus(self) -> int:
        return int(self.bus_id.shape[0])

    @property
    def n_branch(self) -> int:
        return int(self.br_from.shape[0])

    @property
    def n_gen(self) -> int:
        return int(self.gen_bus.shape[0])

    def copy(self) -> "GridModel":
        kw = {k: (v.copy() if isinstance(v, (np.ndarray, dict, list)) else v) for k, v in self.__dict__.items()
              if k != "_keep"}
        return GridModel(**kw)

    def machines(self) -> dict:
        """The units' machine data with the Generator record's defaults where the model gives none (Pmin 0,
        Pmax +inf, MBase 100 MVA, H 0, type "", not power-flow-only, converter flag inferred from the type)."""
        ng = self.n_gen
        pick = lambda a, d, dt: np.full(ng, d, dt) if a is None else np.asarray(a, dt)  # noqa: E731
        return {"pmin": pick(self.pmin, 0.0, np.float64), "pmax": pick(self.pmax, np.inf, np.float64),
                "mbase": pick(self.mbase, 100.0, np.float64), "inertia_h": pick(self.inertia_h, 0.0, np.float64),
                "gen_type": list(self.gen_type) if self.gen_type is not None else [""] * ng,
                "pf_only": pick(self.pf_only, 0, np.uint8), "converter": pick(self.converter, -1, np.int8)}

    def branch_label(self, k: int) -> str:
        """A branch's name, or its end buses "from-to" when it has none (ContingencyAnalysis.cs:1168-1172)."""
        nm = self.br_name[k] if self.br_name is not None else ""
        return nm if nm and nm.strip() else f"{int(self.bus_id[self.br_from[k]])}-{int(self.bus_id[self.br_to[k]])}"

    def boundary_members(self):
        """Boundary members resolved to branch positions: (ptr, branch, direction, limit MW), CSR. Every member name
        must name exactly one branch, and every direction must be 1 or -1 (Boundary.BranchNameProblems,
        Model/Model.cs:535-551; JsonGridLoader.cs:219-223); otherwise ValueError lists the problems."""
        names = self.br_name if self.br_name is not None else [""] * self.n_branch
        where = {}
        for k, nm in enumerate(names):
            if nm:
                where.setdefault(nm, []).append(k)
        ptr, br, dr, lim, bad = [0], [], [], [], []
        for name, limit, members in self.boundaries:
            for bn, d in members:
                ks = where.get(bn, [])
                if len(ks) != 1:
                    bad.append(f"boundary '{name}' names branch '{bn}', which "
                               + ("matches no branch of the case" if not ks else f"{len(ks)} branches share"))
                    continue
                if d not in (1, -1):
                    bad.append(f"boundary '{name}': branch '{bn}' has direction {d}; it must be 1 or -1")
                    continue
                br.append(ks[0])
                dr.append(int(d))
            ptr.append(len(br))
            lim.append(float(limit))
        if bad:
            raise ValueError("; ".join(bad[:20]))
        return (np.array(ptr, np.int32), np.array(br, np.int32), np.array(dr, np.int32), np.array(lim, np.float64))

    def with_voltages(self, vm: np.ndarray, va_deg: np.ndarray) -> "GridModel":
        """Warm start: every bus starts at the given state (GridScenario.WithSolvedVoltages,
        ``src/GridSim.Core/Simulation/GridScenario.cs:35-52``)."""
        m = self.copy()
        m.vm = np.ascontiguousarray(vm, dtype=np.float64).copy()
        m.va_deg = np.ascontiguousarray(va_deg, dtype=np.float64).copy()
        return m

    def flat_started(self) -> "GridModel":
        """The model whose stored voltages are the flat start of PowerFlowOptions.FlatStart: every bus that is not
        a reference bus starts at 1 pu and 0 degrees, a reference bus keeps its stored Vm and angle, and a
        voltage-controlled bus with units still starts at its units' set point (``NewtonShell.cs:463-474``). The
        library takes a flat start this way, through the descriptor."""
        m = self.copy()
        free = m.bus_type != SLACK
        m.vm[free] = 1.0
        m.va_deg[free] = 0.0
        return m

    def in_service_branches(self) -> np.ndarray:
        """ContingencyAnalysis.InServiceBranchIndices (``ContingencyAnalysis.cs:283-289``)."""
        return np.nonzero(self.br_in_service)[0].astype(np.int32)

    def desc(self):
        """A ``gs_grid_desc`` pointing at this model's arrays (kept alive by the model)."""
        from ._abi import GridDesc

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a.ctypes.data_as(ctypes.c_void_p)

        d = GridDesc()
        d.n_bus, d.n_gen, d.n_branch = self.n_bus, self.n_gen, self.n_branch
        d.base_mva = float(self.base_mva)
        d.bus_id = arr(self.bus_id, np.int32)
        d.bus_type = arr(self.bus_type, np.int32)
        d.pd, d.qd = arr(self.pd, np.float64), arr(self.qd, np.float64)
        d.gs, d.bs = arr(self.gs, np.float64), arr(self.bs, np.float64)
        d.vm, d.va_deg = arr(self.vm, np.float64), arr(self.va_deg, np.float64)
        d.vmin_pu, d.vmax_pu = arr(self.vmin, np.float64), arr(self.vmax, np.float64)
        d.gen_bus = arr(self.gen_bus, np.int32)
        d.pg, d.qg, d.vg = arr(self.pg, np.float64), arr(self.qg, np.float64), arr(self.vg, np.float64)
        d.qmin, d.qmax = arr(self.qmin, np.float64), arr(self.qmax, np.float64)
        d.gen_in_service = arr(self.gen_in_service, np.uint8)
        d.br_from, d.br_to = arr(self.br_from, np.int32), arr(self.br_to, np.int32)
        d.r, d.x, d.b = arr(self.r, np.float64), arr(self.x, np.float64), arr(self.b, np.float64)
        d.tap, d.shift_deg = arr(self.tap, np.float64), arr(self.shift_deg, np.float64)
        d.rate_a = arr(self.rate_a, np.float64)
        d.br_in_service = arr(self.br_in_service, np.uint8)
        if self.rate_b is not None:
            d.rate_b = arr(self.rate_b, np.float64)
        if self.rate_c is not None:
            d.rate_c = arr(self.rate_c, np.float64)
        if self.boundaries:
            ptr, br, dr, lim = self.boundary_members()
            d.n_boundary = len(self.boundaries)
            d.bnd_ptr, d.bnd_branch = arr(ptr, np.int32), arr(br, np.int32)
            d.bnd_dir, d.bnd_limit_mw = arr(dr, np.int32), arr(lim, np.float64)
        if self.zip is not None:
            d.zip = arr(np.asarray(self.zip, np.float64).reshape(-1), np.float64)
        return d

    # ---- JSON round trip of the whole model (golden fixtures) -------------------------------------
    def to_dict(self) -> dict:
        out = {"name": self.name, "base_mva": self.base_mva}
        for k, v in self.__dict__.items():
            if isinstance(v, np.ndarray):
                out[k] = [None if (isinstance(t, float) and math.isnan(t)) else t for t in v.tolist()]
        if self.br_name is not None:
            out["br_name"] = list(self.br_name)
        if self.boundaries:
            out["boundaries"] = [[nm, lim, [list(x) for x in mem]] for nm, lim, mem in self.boundaries]
        if self.gen_type is not None:
            out["gen_type"] = list(self.gen_type)
        return out

    @staticmethod
    def from_dict(d: dict) -> "GridModel":
        f64 = lambda k: np.array([np.nan if t is None else t for t in d[k]], dtype=np.float64)  # noqa: E731
        i32 = lambda k: np.array(d[k], dtype=np.int32)  # noqa: E731
        u8 = lambda k: np.array(d[k], dtype=np.uint8)  # noqa: E731
        return GridModel(
            name=d["name"], base_mva=float(d["base_mva"]),
            bus_id=i32("bus_id"), bus_type=i32("bus_type"), pd=f64("pd"), qd=f64("qd"), gs=f64("gs"),
            bs=f64("bs"), vm=f64("vm"), va_deg=f64("va_deg"), vmin=f64("vmin"), vmax=f64("vmax"),
            base_kv=f64("base_kv"), gen_bus=i32("gen_bus"), pg=f64("pg"), qg=f64("qg"), vg=f64("vg"),
            qmin=f64("qmin"), qmax=f64("qmax"), gen_in_service=u8("gen_in_service"), br_from=i32("br_from"),
            br_to=i32("br_to"), r=f64("r"), x=f64("x"), b=f64("b"), tap=f64("tap"), shift_deg=f64("shift_deg"),
            rate_a=f64("rate_a"), br_in_service=u8("br_in_service"), is_transformer=u8("is_transformer"),
            rate_b=f64("rate_b") if "rate_b" in d else None, rate_c=f64("rate_c") if "rate_c" in d else None,
            br_name=list(d["br_name"]) if "br_name" in d else None,
            boundaries=[(nm, float(lim), [(str(b), int(x)) for b, x in mem]) for nm, lim, mem in d.get("boundaries", [])],
            pmin=f64("pmin") if "pmin" in d else None, pmax=f64("pmax") if "pmax" in d else None,
            mbase=f64("mbase") if "mbase" in d else None, inertia_h=f64("inertia_h") if "inertia_h" in d else None,
            gen_type=list(d["gen_type"]) if "gen_type" in d else None,
            pf_only=u8("pf_only") if "pf_only" in d else None,
            converter=np.array(d["converter"], np.int8) if "converter" in d else None,
            zip=np.array(d["zip"], np.float64).reshape(-1, 6) if "zip" in d else None)


# =============================================================================================
# MATPOWER .m (MatpowerParser.cs)

def _matrix(text: str, name: str):
    m = re.search(r"mpc\." + name + r"\s*=\s*\[(.*?)\];", text, re.S)
    if not m:
        return None
    rows = []
    for line in m.group(1).replace("...", " ").split(";"):
        vals = line.split()
        if vals:
            rows.append([float(v) for v in vals])
    return rows


def parse_matpower(text: str, name: str = "matpower") -> GridModel:
    text = re.sub(r"%[^\n]*", "", text)  # comments
    mb = re.search(r"mpc\.baseMVA\s*=\s*([0-9.eE+-]+)", text)
    base = float(mb.group(1)) if mb else 100.0
    bus_rows = _matrix(text, "bus")
    gen_rows = _matrix(text, "gen") or []
    br_rows = _matrix(text, "branch") or []
    buses = [r for r in bus_rows if int(r[1]) != 4]
    live = {int(r[0]) for r in buses}
    pos = {int(r[0]): i for i, r in enumerate(buses)}
    gens = [g for g in gen_rows if int(g[0]) in live]
    gen_on = {int(g[0]) for g in gens if int(g[7]) > 0}
    btype = []
    for r in buses:
        t = {3: SLACK, 2: PV}.get(int(r[1]), PQ)
        if t == PV and int(r[0]) not in gen_on:  # :341-349
            t = PQ
        btype.append(t)

    def limits(r):
        if len(r) >= 13:
            hi, lo = r[11], r[12]
            if math.isfinite(lo) and math.isfinite(hi) and lo > 0 and hi > 0 and lo <= hi:
                return lo, hi
        return math.nan, math.nan

    lim = [limits(r) for r in buses]
    brs = [r for r in br_rows if int(r[10]) != 0 and int(r[0]) in live and int(r[1]) in live]
    g = lambda rows, i, d=0.0: np.array([r[i] if i < len(r) else d for r in rows], dtype=np.float64)  # noqa: E731
    tap_raw = g(brs, 8)
    return GridModel(
        name=name, base_mva=base,
        bus_id=np.array([int(r[0]) for r in buses], np.int32), bus_type=np.array(btype, np.int32),
        pd=g(buses, 2), qd=g(buses, 3), gs=g(buses, 4), bs=g(buses, 5), vm=g(buses, 7, 1.0), va_deg=g(buses, 8),
        vmin=np.array([v[0] for v in lim]), vmax=np.array([v[1] for v in lim]), base_kv=g(buses, 9),
        gen_bus=np.array([pos[int(r[0])] for r in gens], np.int32), pg=g(gens, 1), qg=g(gens, 2),
        vg=g(gens, 5, 1.0), qmin=g(gens, 4, -np.inf), qmax=g(gens, 3, np.inf),
        gen_in_service=np.array([1 if int(r[7]) > 0 else 0 for r in gens], np.uint8),
        br_from=np.array([pos[int(r[0])] for r in brs], np.int32),
        br_to=np.array([pos[int(r[1])] for r in brs], np.int32),
        r=g(brs, 2), x=g(brs, 3), b=g(brs, 4), tap=np.where(tap_raw != 0.0, tap_raw, 1.0), shift_deg=g(brs, 9),
        rate_a=g(brs, 5), br_in_service=np.ones(len(brs), np.uint8),
        is_transformer=(tap_raw != 0.0).astype(np.uint8),
        rate_b=g(brs, 6), rate_c=g(brs, 7),  # RATE_B / RATE_C (MatpowerParser.cs:384-385)
        # PMIN / PMAX / MBASE, a zero MBASE replaced by the system base, H 0 (MatpowerParser.cs:272-307)
        pmin=g(gens, 9), pmax=g(gens, 8, np.inf), mbase=np.where(g(gens, 6) > 0, g(gens, 6), base),
        inertia_h=np.zeros(len(gens)))


def load_matpower(path: str) -> GridModel:
    with open(path) as fh:
        return parse_matpower(fh.read(), os.path.splitext(os.path.basename(path))[0])


# =============================================================================================
# GridSim v1 JSON case directory (JsonGridLoader.cs:55-255), the subset this path uses.

def save_case_dir(m: GridModel, path: str) -> None:
    os.makedirs(path, exist_ok=True)
    tname = {PQ: "pq", PV: "pv", SLACK: "slack"}

    def dump(fn, obj):
        with open(os.path.join(path, fn), "w") as fh:
            json.dump(obj, fh, indent=1)

    dump("system.json", {"name": m.name, "baseMva": m.base_mva, "frequencyHz": 50.0, "dispatch": False})
    buses = []
    for i in range(m.n_bus):
        d = {"id": int(m.bus_id[i]), "type": tname[int(m.bus_type[i])], "baseKv": float(m.base_kv[i]),
             "vm": float(m.vm[i]), "vaDeg": float(m.va_deg[i]), "gs": float(m.gs[i]), "bs": float(m.bs[i])}
        if not math.isnan(m.vmin[i]):
            d["vminPu"] = float(m.vmin[i])
        if not math.isnan(m.vmax[i]):
            d["vmaxPu"] = float(m.vmax[i])
        if m.zip is not None and zip_varies(m.zip[i]):
            d["zip"] = dict(zip(("ap", "bp", "cp", "aq", "bq", "cq"), (float(c) for c in m.zip[i])))
        buses.append(d)
    dump("buses.json", buses)
    gens = []
    mach = m.machines()
    for k in range(m.n_gen):
        bi = int(m.gen_bus[k])
        # capacityMva is the unit's MBase when the model has machine data (JsonGridLoader.cs:166)
        cap = (float(mach["mbase"][k]) if m.mbase is not None and mach["mbase"][k] > 0
               else float(max(abs(m.qmax[k]), abs(m.qmin[k]), abs(m.pg[k]), 1.0)))
        g = {"name": f"G{k}", "bus": int(m.bus_id[bi]), "role": "slack" if m.bus_type[bi] == SLACK else "pv",
             "capacityMva": cap, "outputMw": float(m.pg[k]), "qOutputMvar": float(m.qg[k]),
             "voltageSetpoint": float(m.vg[k]), "qMinMvar": float(m.qmin[k]), "qMaxMvar": float(m.qmax[k]),
             "inService": bool(m.gen_in_service[k]), "pMinMw": float(mach["pmin"][k]),
             "pMaxMw": float(mach["pmax"][k]), "inertiaH": float(mach["inertia_h"][k])}
        if mach["gen_type"][k]:
            g["type"] = mach["gen_type"][k]
        if mach["pf_only"][k]:
            g["powerFlowOnly"] = True
        if mach["converter"][k] >= 0:
            g["converterInterfaced"] = bool(mach["converter"][k])
        gens.append(g)
    dump("generation.json", gens)
    dump("demand.json", [{"name": f"D{i}", "bus": int(m.bus_id[i]), "pMw": float(m.pd[i]), "qMvar": float(m.qd[i])}
                         for i in range(m.n_bus) if m.pd[i] != 0 or m.qd[i] != 0])
    lines = []
    for k in range(m.n_branch):
        ln = {"name": m.br_name[k] if m.br_name is not None and m.br_name[k] else f"L{k}",
              "from": int(m.bus_id[m.br_from[k]]), "to": int(m.bus_id[m.br_to[k]]),
              "rPu": float(m.r[k]), "xPu": float(m.x[k]), "bPu": float(m.b[k]),
              "ratingMva": float(m.rate_a[k]), "tapRatio": float(m.tap[k]),
              "phaseShiftDeg": float(m.shift_deg[k]), "isTransformer": bool(m.is_transformer[k])}
        for key, arr in (("ratingBMva", m.rate_b), ("ratingCMva", m.rate_c)):
            if arr is not None and arr[k] != 0:
                ln[key] = float(arr[k])
        lines.append(ln)
    dump("transmission.json", lines)
    if m.boundaries:
        dump("boundaries.json", [{"name": nm, "limitMw": lim,
                                  "branches": [{"branch": b, "direction": d} for b, d in mem]}
                                 for nm, lim, mem in m.boundaries])


def load_case_dir(path: str) -> GridModel:
    def read(fn, default):
        p = os.path.join(path, fn)
        if not os.path.exists(p):
            return default
        with open(p) as fh:
            return json.load(fh)

    sysd = read("system.json", {})
    buses = read("buses.json", [])
    gens = read("generation.json", [])
    dem = read("demand.json", [])
    lines = read("transmission.json", [])
    txs = read("transformer.json", [])
    bnds = read("boundaries.json", [])
    if not buses:
        raise ValueError("buses.json is empty or missing")
    if sysd.get("dispatch", True):
        raise ValueError("only cases with \"dispatch\": false are read (the written outputs are the dispatch)")
    pos = {int(b["id"]): i for i, b in enumerate(buses)}
    n = len(buses)
    btype = np.array([{"pq": PQ, "pv": PV, "slack": SLACK}[b.get("type", "pq").lower()] for b in buses], np.int32)
    for g in gens:  # JsonGridLoader.cs:121-127: generator roles raise bus types
        if not g.get("inService", True):
            continue
        i = pos[int(g["bus"])]
        role = g.get("role", "pv").lower()
        if role == "slack":
            btype[i] = SLACK
        elif role != "pq" and btype[i] != SLACK:
            btype[i] = PV
    pd = np.zeros(n)
    qd = np.zeros(n)
    for d in dem:
        i = pos[int(d["bus"])]
        pd[i] += d["pMw"]
        qd[i] += d["qMvar"] if d.get("qMvar") is not None else d["pMw"] * math.tan(math.acos(d.get("powerFactor", 0.95)))
    f = lambda rows, k, dflt=0.0: np.array([float(r.get(k, dflt)) if r.get(k) is not None else dflt  # noqa: E731
                                           for r in rows], np.float64)
    circ = np.array([int(l.get("circuits", 1)) for l in lines], np.float64)
    if (circ < 1).any():
        raise ValueError("a line has circuits below 1")
    cap = f(gens, "capacityMva")
    # transformers follow the lines as branches (JsonGridLoader.cs:189-196): no charging, ratings per unit
    ntx = len(txs)
    cat = lambda a, b: np.concatenate([a, b])  # noqa: E731
    one = np.ones(ntx)
    return GridModel(
        name=sysd.get("name", os.path.basename(os.path.normpath(path))), base_mva=float(sysd.get("baseMva", 100.0)),
        bus_id=np.array([int(b["id"]) for b in buses], np.int32), bus_type=btype, pd=pd, qd=qd,
        gs=f(buses, "gs"), bs=f(buses, "bs"), vm=f(buses, "vm", 1.0), va_deg=f(buses, "vaDeg"),
        vmin=f(buses, "vminPu", math.nan), vmax=f(buses, "vmaxPu", math.nan), base_kv=f(buses, "baseKv"),
        gen_bus=np.array([pos[int(g["bus"])] for g in gens], np.int32), pg=f(gens, "outputMw"),
        qg=f(gens, "qOutputMvar"), vg=f(gens, "voltageSetpoint", 1.0),
        qmin=np.array([g["qMinMvar"] if g.get("qMinMvar") is not None else -c for g, c in zip(gens, cap)], np.float64),
        qmax=np.array([g["qMaxMvar"] if g.get("qMaxMvar") is not None else c for g, c in zip(gens, cap)], np.float64),
        gen_in_service=np.array([1 if g.get("inService", True) else 0 for g in gens], np.uint8),
        br_from=np.array([pos[int(l["from"])] for l in lines + txs], np.int32),
        br_to=np.array([pos[int(l["to"])] for l in lines + txs], np.int32),
        r=cat(f(lines, "rPu") / circ, f(txs, "rPu")), x=cat(f(lines, "xPu") / circ, f(txs, "xPu")),
        b=cat(f(lines, "bPu") * circ, np.zeros(ntx)), tap=cat(f(lines, "tapRatio", 1.0), f(txs, "tapRatio", 1.0)),
        shift_deg=cat(f(lines, "phaseShiftDeg"), f(txs, "phaseShiftDeg")),
        rate_a=cat(f(lines, "ratingMva") * circ, f(txs, "ratingMva")),
        br_in_service=np.ones(len(lines) + ntx, np.uint8),
        is_transformer=np.array([1 if l.get("isTransformer", False) else 0 for l in lines] + [1] * ntx, np.uint8),
        zip=_json_zip(buses),
        rate_b=cat(f(lines, "ratingBMva") * circ, f(txs, "ratingBMva") * one),
        rate_c=cat(f(lines, "ratingCMva") * circ, f(txs, "ratingCMva") * one),
        br_name=[l.get("name") or "" for l in lines + txs],
        # machine data (JsonGridLoader.cs:158-170): Pmin 0 and Pmax capacityMva unless written, MBase capacityMva
        pmin=f(gens, "pMinMw"), pmax=np.array([float(g["pMaxMw"]) if g.get("pMaxMw") is not None else c
                                               for g, c in zip(gens, cap)], np.float64),
        mbase=cap.copy(), inertia_h=f(gens, "inertiaH"),
        gen_type=[g.get("type") if g.get("type") is not None else "ccgt" for g in gens],
        pf_only=np.array([1 if g.get("powerFlowOnly", False) else 0 for g in gens], np.uint8),
        converter=np.array([-1 if g.get("converterInterfaced") is None else int(bool(g["converterInterfaced"]))
                            for g in gens], np.int8),
        boundaries=[(b.get("name", ""), float(b.get("limitMw", 0.0)),
                     [(x.get("branch", ""), int(x.get("direction", 1))) for x in (b.get("branches") or [])])
                    for b in bnds])
