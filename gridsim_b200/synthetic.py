"""Seeded synthetic transmission grids of the benchmark workloads.

Construction (one rule set for every size, PCG64 seeded):

* topology: ``n`` points uniform in the unit square; the Euclidean minimum spanning tree (over the
  Delaunay triangulation) plus nearest-neighbour non-tree edges, no duplicates, until there are
  ``n_branch`` branches, taken longest tree detour first (the chains of the tree are meshed first);
* 10 % of the branches are transformers with tap U(0.95, 1.05), no phase shift and no charging, and a
  leakage reactance X U(0.05, 0.15) pu with R = X / U(3, 10);
* lines: series R U(0.001, 0.05) pu, X = R * U(3, 10), charging B U(0, 0.1) pu;
* one slack (the bus nearest the centre) and ``n_pv`` PV buses drawn uniformly; voltage set points are
  uniform on [0.98, 1.05] but spatially smooth (neighbouring units hold neighbouring set points);
* loads on every non-generator bus, P lognormal (median 0.3 pu, sigma 0.8), power factor U(0.9, 0.98)
  lagging; generation splits 1.02 x total load over the PV buses in proportion to U(0.5, 1.5) times the
  load of each unit's Voronoi cell (so that generation sits near load); the slack takes the rest and
  the losses;
* generous reactive limits (10 x capacity) so they never bind; own voltage limits 0.95-1.05 pu;
* thermal ratings U(1.2, 2.0) x the base-case branch flow max(|S_f|, |S_t|), floor 1 MVA.

The data layout is that of the reference's GridModel (``gridsim_b200.model.GridModel``); use
``gridsim_b200.model.save_case_dir`` to write it as a GridSim v1 JSON case directory with
``"dispatch": false``.
"""
from __future__ import annotations

import math

import numpy as np

from .model import PQ, PV, SLACK, GridModel

# Sizes of the benchmark workloads (bus count, branch count, PV count).
CONFIG_SIZES = {
    0: (120, 180, 20),
    1: (2000, 2800, 250),
    2: (10000, 13500, 1200),
}


def _edges(pts: np.ndarray, n_branch: int, rng: np.random.Generator) -> np.ndarray:
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import minimum_spanning_tree
    from scipy.spatial import Delaunay, cKDTree

    n = pts.shape[0]
    tri = Delaunay(pts)
    s = tri.simplices
    e = np.concatenate([s[:, [0, 1]], s[:, [1, 2]], s[:, [0, 2]]])
    e = np.unique(np.sort(e, axis=1), axis=0)
    w = np.linalg.norm(pts[e[:, 0]] - pts[e[:, 1]], axis=1)
    mst = minimum_spanning_tree(coo_matrix((w, (e[:, 0], e[:, 1])), shape=(n, n))).tocoo()
    tree = np.sort(np.stack([mst.row, mst.col], 1), axis=1)
    have = {(int(a), int(b)) for a, b in tree}
    edges = [tuple(t) for t in tree.tolist()]
    # Candidate extra branches: each bus's nearest neighbours (no duplicates, no tree branch). They are taken
    # in order of the tree detour they close (hops along the spanning tree between their ends, longest
    # first; shorter branch first among equals): the long chains of the tree are meshed first, as grid
    # planners reinforce the weakest corridors, instead of adding loops inside dense clusters.
    depth, up = _tree_lifting(n, tree)
    k = 8
    while True:
        d, nb = cKDTree(pts).query(pts, k=min(k + 1, n))
        a = np.repeat(np.arange(n), nb.shape[1] - 1)
        b = nb[:, 1:].ravel()
        dist = d[:, 1:].ravel()
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        key = lo.astype(np.int64) * n + hi
        _, first = np.unique(key, return_index=True)
        lo, hi, dist = lo[first], hi[first], dist[first]
        fresh = np.array([(int(x), int(y)) not in have for x, y in zip(lo, hi)], bool)
        lo, hi, dist = lo[fresh], hi[fresh], dist[fresh]
        if lo.shape[0] + len(edges) >= n_branch or k >= n - 1:
            break
        k *= 2
    hops = _tree_hops(lo, hi, depth, up)
    order = np.lexsort((dist, -hops))
    for j in order[: max(0, n_branch - len(edges))]:
        edges.append((int(lo[j]), int(hi[j])))
    out = np.array(edges[:n_branch], dtype=np.int64)
    return out[rng.permutation(out.shape[0])]  # branch order independent of construction order


def _tree_lifting(n: int, tree: np.ndarray):
    """Depths and binary-lifting ancestor tables of a spanning tree rooted at bus 0."""
    from collections import deque
    adj = [[] for _ in range(n)]
    for a, b in tree:
        adj[int(a)].append(int(b))
        adj[int(b)].append(int(a))
    parent = np.zeros(n, np.int64)
    depth = np.zeros(n, np.int64)
    seen = np.zeros(n, bool)
    seen[0] = True
    dq = deque([0])
    while dq:
        u = dq.popleft()
        for v in adj[u]:
            if not seen[v]:
                seen[v] = True
                parent[v] = u
                depth[v] = depth[u] + 1
                dq.append(v)
    up = [parent]
    for _ in range(max(1, int(depth.max()).bit_length())):
        up.append(up[-1][up[-1]])
    return depth, up


def _tree_hops(a: np.ndarray, b: np.ndarray, depth: np.ndarray, up) -> np.ndarray:
    """Hop distance along the tree between bus pairs (vectorised lowest common ancestor)."""
    a = a.astype(np.int64).copy()
    b = b.astype(np.int64).copy()
    swap = depth[a] < depth[b]
    a[swap], b[swap] = b[swap], a[swap]
    diff = depth[a] - depth[b]
    x = a.copy()
    for j, u in enumerate(up):
        sel = ((diff >> j) & 1).astype(bool)
        x[sel] = u[x[sel]]
    y = b.copy()
    for u in reversed(up):
        sel = u[x] != u[y]
        x[sel] = u[x[sel]]
        y[sel] = u[y[sel]]
    lca = np.where(x == y, x, up[0][x])
    return depth[a] + depth[b] - 2 * depth[lca]


def _smooth_uniform(n: int, e: np.ndarray, rng: np.random.Generator, lo: float, hi: float, sweeps: int = 30):
    """A spatially smooth field over the buses whose values are uniform on [lo, hi]: white noise averaged
    over graph neighbourhoods, then rank-mapped to evenly spaced quantiles. Neighbouring generators get
    neighbouring voltage set points, as real set points follow the voltage profile."""
    import scipy.sparse as sp
    z = rng.standard_normal(n)
    a = sp.coo_matrix((np.ones(2 * e.shape[0]), (np.r_[e[:, 0], e[:, 1]], np.r_[e[:, 1], e[:, 0]])), shape=(n, n)).tocsr()
    deg = np.asarray(a.sum(axis=1)).ravel() + 1.0
    for _ in range(sweeps):
        z = (z + a @ z) / deg
    ranks = np.empty(n)
    ranks[np.argsort(z, kind="stable")] = (np.arange(n) + rng.uniform(0.0, 1.0, size=n)) / n
    return lo + (hi - lo) * ranks


def _nearest_source(n: int, e: np.ndarray, sources: np.ndarray) -> np.ndarray:
    """For every bus, the index (into `sources`) of the source fewest branch hops away."""
    from collections import deque
    adj = [[] for _ in range(n)]
    for a, b in e:
        adj[int(a)].append(int(b))
        adj[int(b)].append(int(a))
    owner = np.full(n, -1, np.int64)
    dq = deque()
    for k, s in enumerate(sources):
        owner[int(s)] = k
        dq.append(int(s))
    while dq:
        u = dq.popleft()
        for v in adj[u]:
            if owner[v] < 0:
                owner[v] = owner[u]
                dq.append(v)
    owner[owner < 0] = 0
    return owner


def _dc_angles(n: int, f: np.ndarray, t: np.ndarray, x: np.ndarray, p_pu: np.ndarray, slack: int) -> np.ndarray:
    """DC load-flow angles (radians) with the slack at 0."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    bs = 1.0 / x
    B = sp.coo_matrix((np.concatenate([bs, bs, -bs, -bs]), (np.concatenate([f, t, f, t]), np.concatenate([f, t, t, f]))),
                      shape=(n, n)).tocsr()
    keep = np.r_[0:slack, slack + 1:n]
    th = np.zeros(n)
    th[keep] = sla.spsolve(B[keep][:, keep].tocsc(), p_pu[keep])
    return th


R_MIN = 0.001


# ---------------------------------------------------------------------------------------------
# Operating point by continuation. The stated element data (uniform independent set points, off-nominal
# taps on branches down to X = 0.003 pu, charging up to 0.1 pu, heavy-tailed loads on a tree-like grid)
# give cases that a damped Newton iteration cannot solve from a flat or DC start at 2,000 buses and
# above. So the case's start point is found by continuation: at a light load, taps and voltage set
# points are ramped from 1 towards their drawn values (as far as a solution exists: the fraction reached
# is kept); then the load (and the generation and charging that follow it) is ramped up as far as a
# solution exists. The stored case is the last solved load level times
# OPERATING_MARGIN, with that state as every bus's start voltage (a case file's stored voltages),
# so the reference engine solves it from its stored start.

OPERATING_MARGIN = 0.6
_LIGHT_LOAD = 0.001


def _ybus(m: GridModel, tap: np.ndarray, bscale: float):
    import scipy.sparse as sp
    n, f, t = m.n_bus, m.br_from, m.br_to
    ys = 1.0 / (m.r + 1j * m.x)
    bc = 1j * m.b * bscale / 2.0
    a = tap * np.exp(1j * np.deg2rad(m.shift_deg))
    vals = np.concatenate([(ys + bc) / (np.abs(a) ** 2), ys + bc, -ys / np.conj(a), -ys / a])
    Y = sp.coo_matrix((vals, (np.concatenate([f, t, f, t]), np.concatenate([f, t, t, f]))), shape=(n, n)).tocsr()
    return Y + sp.diags((m.gs + 1j * m.bs) / m.base_mva)


def _newton(Y, sbus: np.ndarray, V: np.ndarray, pv: np.ndarray, pq: np.ndarray, tol=1e-9, maxit=25):
    """Complex-form polar Newton with the reference's step damping (largest correction 0.4)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    pvpq = np.r_[pv, pq]
    npv = pvpq.shape[0]
    V = V.copy()
    for _ in range(maxit + 1):
        mis = V * np.conj(Y @ V) - sbus
        F = np.r_[mis[pvpq].real, mis[pq].imag]
        if not np.all(np.isfinite(F)):
            return None
        if np.abs(F).max() < tol:
            return V
        Ib = Y @ V
        dV = sp.diags(V)
        Vn = sp.diags(V / np.abs(V))
        dS_dVm = dV @ np.conj(Y @ Vn) + sp.diags(np.conj(Ib)) @ Vn
        dS_dVa = 1j * dV @ np.conj(sp.diags(Ib) - Y @ dV)
        J = sp.bmat([[dS_dVa[pvpq][:, pvpq].real, dS_dVm[pvpq][:, pq].real],
                     [dS_dVa[pq][:, pvpq].imag, dS_dVm[pq][:, pq].imag]]).tocsc()
        try:
            dx = -sla.spsolve(J, F)
        except Exception:
            return None
        if not np.all(np.isfinite(dx)):
            return None
        mx = np.abs(dx).max()
        dx *= 0.4 / mx if mx > 0.4 else 1.0
        va = np.angle(V)
        vm = np.abs(V)
        va[pvpq] += dx[:npv]
        vm[pq] = np.maximum(vm[pq] + dx[npv:], 0.01)
        V = vm * np.exp(1j * va)
    return None


def find_operating_point(m: GridModel, margin: float = OPERATING_MARGIN) -> GridModel:
    """Scale the load to a solvable level by continuation and store the solved state as the start point: the last
    solvable load level times `margin` (0.6 for the benchmark grids; closer to 1 gives a stressed grid, whose
    outages need more Newton iterations and fail more often)."""
    slack = np.nonzero(m.bus_type == SLACK)[0]
    pv = np.nonzero(m.bus_type == PV)[0]
    pq = np.nonzero(m.bus_type == PQ)[0]
    vg_bus = np.ones(m.n_bus)
    vg_bus[m.gen_bus] = m.vg

    def sbus(lam):
        s = -(m.pd + 1j * m.qd) * lam / m.base_mva
        np.add.at(s, m.gen_bus, (m.pg + 1j * m.qg) * lam / m.base_mva)
        return s

    def state(vm_set):
        v = np.ones(m.n_bus, complex)
        v[m.bus_type != PQ] = vm_set[m.bus_type != PQ]
        return v

    # phase 1: taps and set points from 1 to their values at light load (charging scales with the load)
    V = state(np.ones(m.n_bus))
    s, ds = 0.0, 0.25
    while s < 1.0:
        s_try = min(1.0, s + ds)
        tap = 1.0 + s_try * (m.tap - 1.0)
        vset = 1.0 + s_try * (vg_bus - 1.0)
        V0 = V.copy()
        V0[m.bus_type != PQ] = np.abs(vset[m.bus_type != PQ]) * np.exp(1j * np.angle(V0[m.bus_type != PQ]))
        Vn = _newton(_ybus(m, tap, _LIGHT_LOAD), sbus(_LIGHT_LOAD), V0, pv, pq)
        if Vn is None:
            ds *= 0.5
            if ds < 1e-3:
                break  # the drawn taps and set points have no solution: keep the largest fraction that has
            continue
        V, s = Vn, s_try
        ds = min(ds * 1.5, 0.5)
    tap_s = s
    taps = 1.0 + tap_s * (m.tap - 1.0)
    vg_s = 1.0 + tap_s * (m.vg - 1.0)
    # phase 2: load (and charging) up, geometric steps, as far as a solution exists
    Y1 = None
    lam, V_at = _LIGHT_LOAD, {_LIGHT_LOAD: V}
    step = 1.5
    while lam < 1.0:
        lam_try = min(1.0, lam * step)
        Vn = _newton(_ybus(m, taps, lam_try), sbus(lam_try), V, pv, pq)
        if Vn is None:
            step = 1.0 + (step - 1.0) * 0.5
            if step < 1.01:
                break
            continue
        V, lam = Vn, lam_try
        V_at[lam] = V
    final = lam if lam >= 1.0 else lam * margin
    if final != lam:
        Vf = _newton(_ybus(m, taps, final), sbus(final), V, pv, pq)
        if Vf is None:
            final = max(k for k in V_at if k <= final) if any(k <= final for k in V_at) else lam
            Vf = V_at.get(final, V)
        V = Vf
    del Y1
    out = m.copy()
    out.pd, out.qd, out.pg, out.qg, out.b = m.pd * final, m.qd * final, m.pg * final, m.qg * final, m.b * final
    out.qmin, out.qmax = m.qmin * max(final, 1e-3), m.qmax * max(final, 1e-3)
    out.tap = taps
    out.vg = vg_s
    out.vm = np.abs(V)
    out.va_deg = np.degrees(np.angle(V) - np.angle(V[slack[0]]))
    out.meta = dict(m.meta, load_scale=final, tap_setpoint_scale=tap_s)
    # thermal ratings from the solved base state: U(1.2, 2.0) x max(|S_f|, |S_t|), floor 1 MVA
    ys = 1.0 / (out.r + 1j * out.x)
    bc = 1j * out.b / 2.0
    a = out.tap * np.exp(1j * np.deg2rad(out.shift_deg))
    vf, vt = V[out.br_from], V[out.br_to]
    i_f = (ys + bc) / np.abs(a) ** 2 * vf - ys / np.conj(a) * vt
    i_t = -ys / a * vf + (ys + bc) * vt
    flow = np.maximum(np.abs(vf * np.conj(i_f)), np.abs(vt * np.conj(i_t))) * out.base_mva
    rng = np.random.Generator(np.random.PCG64(int(m.meta.get("seed", 0)) + 7919))
    out.rate_a = np.maximum(rng.uniform(1.2, 2.0, size=out.n_branch) * flow, 1.0)
    return out


def make_grid(n_bus: int, n_branch: int, n_pv: int, seed: int, name: str | None = None,
              operating_point: bool = True, margin: float = OPERATING_MARGIN) -> GridModel:
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = rng.uniform(0.0, 1.0, size=(n_bus, 2))
    e = _edges(pts, n_branch, rng)
    nb = e.shape[0]
    base = 100.0

    slack = int(np.argmin(np.linalg.norm(pts - 0.5, axis=1)))
    others = np.array([i for i in range(n_bus) if i != slack])
    pv = np.sort(rng.choice(others, size=n_pv, replace=False))
    btype = np.full(n_bus, PQ, np.int32)
    btype[pv] = PV
    btype[slack] = SLACK
    vg_bus = _smooth_uniform(n_bus, e, rng, 0.98, 1.05)

    is_gen = btype != PQ
    p_load = np.where(is_gen, 0.0, np.exp(np.log(0.3) + 0.8 * rng.standard_normal(n_bus))) * base
    pf = rng.uniform(0.9, 0.98, size=n_bus)
    q_load = p_load * np.tan(np.arccos(pf))
    total = float(p_load.sum())
    wts = rng.uniform(0.5, 1.5, size=n_pv)  # drawn for stream compatibility; see the balance below
    # Each unit supplies the load of its cell (the loads fewer branch hops from it than from any other unit,
    # multi-source breadth-first search), so the grid carries regional flows. Random per-unit weights would
    # leave every cell unbalanced, and with a single slack those imbalances add up across the whole grid
    # (flows of tens of pu on 10k buses: no load flow solution exists).
    near = _nearest_source(n_bus, e, pv)
    cell = np.bincount(near, weights=p_load, minlength=n_pv)
    pg_pv = cell.copy()
    del wts
    gen_bus = np.concatenate([[slack], pv]).astype(np.int32)
    pg = np.concatenate([[0.0], pg_pv])
    cap = np.maximum(np.abs(pg), 0.1 * total / max(n_pv, 1))
    cap[0] = max(total, 1.0)
    vg = vg_bus[gen_bus]

    n_tx = int(round(0.1 * nb))
    tx = np.zeros(nb, bool)
    tx[rng.choice(nb, size=n_tx, replace=False)] = True
    r = rng.uniform(R_MIN, 0.05, size=nb)
    x = r * rng.uniform(3.0, 10.0, size=nb)
    # Transformers carry a leakage reactance U(0.05, 0.15) pu with the same X/R rule: an off-nominal tap on
    # a branch of X = 0.003 pu drives circulating flows of tens of pu round every loop it closes.
    x_tx = rng.uniform(0.05, 0.15, size=nb)
    x = np.where(tx, x_tx, x)
    r = np.where(tx, x_tx / rng.uniform(3.0, 10.0, size=nb), r)
    bch = np.where(tx, 0.0, rng.uniform(0.0, 0.1, size=nb))
    tap = np.where(tx, rng.uniform(0.95, 1.05, size=nb), 1.0)

    m = GridModel(
        name=name or f"synthetic-{n_bus}-s{seed}", base_mva=base,
        bus_id=np.arange(1, n_bus + 1, dtype=np.int32), bus_type=btype, pd=p_load, qd=q_load,
        gs=np.zeros(n_bus), bs=np.zeros(n_bus), vm=np.where(is_gen, vg_bus, 1.0), va_deg=np.zeros(n_bus),
        vmin=np.full(n_bus, 0.95), vmax=np.full(n_bus, 1.05), base_kv=np.full(n_bus, 230.0),
        gen_bus=gen_bus, pg=pg, qg=np.zeros(gen_bus.shape[0]), vg=vg, qmin=-10.0 * cap, qmax=10.0 * cap,
        gen_in_service=np.ones(gen_bus.shape[0], np.uint8),
        br_from=e[:, 0].astype(np.int32), br_to=e[:, 1].astype(np.int32), r=r, x=x, b=bch, tap=tap,
        shift_deg=np.zeros(nb), rate_a=np.zeros(nb), br_in_service=np.ones(nb, np.uint8),
        is_transformer=tx.astype(np.uint8), meta={"seed": seed})
    return find_operating_point(m, margin) if operating_point else m


def config_grid(config: int, seed: int = 0, margin: float = OPERATING_MARGIN) -> GridModel:
    """The grid of a benchmark configuration; `margin` other than 0.6 gives its stressed variant (same topology,
    parameters and outage sets, the operating point at that share of the last solvable load level)."""
    n, b, p = CONFIG_SIZES[config]
    suffix = "" if margin == OPERATING_MARGIN else f"-m{margin:g}"
    return make_grid(n, b, p, seed, name=f"synthetic-config{config}-{n}bus-s{seed}{suffix}", margin=margin)


def bridges(m: GridModel) -> np.ndarray:
    """Mask of in-service branches whose removal disconnects the grid (iterative Tarjan)."""
    n = m.n_bus
    adj = [[] for _ in range(n)]
    for k in range(m.n_branch):
        if m.br_in_service[k]:
            a, b = int(m.br_from[k]), int(m.br_to[k])
            adj[a].append((b, k))
            adj[b].append((a, k))
    disc = [-1] * n
    low = [0] * n
    is_bridge = np.zeros(m.n_branch, bool)
    t = 0
    for root in range(n):
        if disc[root] >= 0:
            continue
        disc[root] = low[root] = t
        t += 1
        stack = [(root, -1, iter(adj[root]))]
        while stack:
            u, pe, it = stack[-1]
            advanced = False
            for v, k in it:
                if k == pe:
                    continue
                if disc[v] < 0:
                    disc[v] = low[v] = t
                    t += 1
                    stack.append((v, k, iter(adj[v])))
                    advanced = True
                    break
                low[u] = min(low[u], disc[v])
            if not advanced:
                stack.pop()
                if stack:
                    p = stack[-1][0]
                    low[p] = min(low[p], low[u])
                    if low[u] > disc[p]:
                        is_bridge[pe] = True
    return is_bridge


def outage_set(m: GridModel, count: int | None, seed: int) -> np.ndarray:
    """Every non-bridge in-service branch (count None), or `count` of them sampled without replacement."""
    cand = np.nonzero((~bridges(m)) & (m.br_in_service != 0))[0].astype(np.int32)
    if count is None or count >= cand.shape[0]:
        return cand
    rng = np.random.Generator(np.random.PCG64(seed + 104729))
    return np.sort(rng.choice(cand, size=count, replace=False)).astype(np.int32)


def load_scalings(m: GridModel, count: int, seed: int) -> np.ndarray:
    """Per-case load multipliers: a global U(0.7, 1.3) times per-bus lognormal(sigma 0.05), [count, n_bus]."""
    rng = np.random.Generator(np.random.PCG64(seed + 15485863))
    g = rng.uniform(0.7, 1.3, size=(count, 1))
    return g * np.exp(0.05 * rng.standard_normal((count, m.n_bus)))


def population_specs(n_grids: int = 64, seed: int = 0, lo: int = 100, hi: int = 25000):
    """(n_bus, n_branch, n_pv, seed, name) of the uneven population: bus counts log-uniform in [lo, hi],
    b ~ U(1.35, 1.4) n, n_pv = 0.12 n."""
    rng = np.random.Generator(np.random.PCG64(seed + 32452843))
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_grids)).astype(int)
    out = []
    for g, n in enumerate(sizes):
        b = int(round(n * rng.uniform(1.35, 1.4)))
        out.append((int(n), b, max(1, int(round(0.12 * n))), seed * 1000 + g, f"synthetic-uneven-{g}-{n}bus"))
    return out


def _make_from_spec(spec):
    n, b, npv, sd, name = spec
    return make_grid(n, b, npv, sd, name=name)


def uneven_population(n_grids: int = 64, seed: int = 0, lo: int = 100, hi: int = 25000, workers: int = 0):
    """The uneven-size population (population_specs), built on `workers` spawned processes (0: in this one)."""
    specs = population_specs(n_grids, seed, lo, hi)
    if workers <= 1:
        return [_make_from_spec(s) for s in specs]
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    order = sorted(range(len(specs)), key=lambda k: -specs[k][0])  # largest first: the pool finishes together
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        built = dict(zip(order, ex.map(_make_from_spec, [specs[k] for k in order])))
    return [built[k] for k in range(len(specs))]
