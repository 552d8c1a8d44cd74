"""Sharding the N-1 screen over ranks (one process per GPU).

The outages of a screen are independent, so each rank screens a shard of them on its own GPU and the per-outage
results are gathered (an all-gather of the compact result records, a few tens of bytes per outage plus the
violation list; no collective runs on the data path) and put back in the caller's row order. The reference
screens outages with a thread pool instead (ContingencyAnalysis.ScreenBranchesParallel,
``src/GridSim.Core/Analysis/ContingencyAnalysis.cs:323-344``); results come back in branch order either way.

Shards are either contiguous count splits (:func:`shard`) or cost-balanced (:func:`balanced_shards`): rows are
dealt by estimated device work, estimated Newton iterations x the per-system LU work. One call screens one grid,
so the LU work is a common factor and the estimate is the iteration count alone (:func:`outage_costs`).
"""
from __future__ import annotations

import heapq
from typing import Callable, Optional, Sequence

import numpy as np

PER_OUTAGE = ("status", "iterations", "max_mismatch", "min_vm", "max_vm", "max_loading_pct")
OPTIONAL = ("worst_boundary_pct", "islanded", "share_notes")  # merged when every part has them

# Estimated Newton iterations of a warm-started outage from the DC flow (pu) the outage removes: 2.3 + 7 x flow,
# fitted on the deciles of the oracle's iteration counts over 1,000 outages of the synthetic 10,000-bus grid
# (mean 2.26 iterations at 0.002 pu, 2.56 at 0.02, 3.07 at 0.08, 3.72 at 0.2; the outages that reach the cap sit
# in the top decile).
ITER_BASE = 2.3
ITER_PER_PU = 7.0


def shard(n_items: int, rank: int, world: int) -> slice:
    """Contiguous balanced split: the first n % world ranks get one item more."""
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def _branch_flows(model) -> np.ndarray:
    """|DC flow| (pu) of every branch at the model's stored angles: |theta_f - theta_t - shift| / x; 0 out of
    service."""
    th = np.radians(np.asarray(model.va_deg, np.float64))
    x = np.where(np.abs(model.x) > 1e-12, np.abs(model.x), 1e-12)
    f = np.abs(th[model.br_from] - th[model.br_to] - np.radians(model.shift_deg)) / x
    return np.where(np.asarray(model.br_in_service) != 0, f, 0.0)


def outage_costs(model, rows, kind: str = "branch", max_iterations: int = 20) -> np.ndarray:
    """Estimated device work of each outage row, in Newton iterations (capped at `max_iterations`).

    kind "branch": rows are branch indices; "sets": rows are [n, k] branch sets (-1 = none), the flows of the set
    summed; "elements": rows are (kind, index) pairs as ``gs_element_screen`` takes them (0 branch, 1 generator
    position, 2 bus position), a generator's removed power its output, a bus's the flows of its branches plus its
    load."""
    flows = _branch_flows(model)
    r = np.asarray(rows)
    if kind == "branch":
        lost = flows[r.astype(np.int64)]
    elif kind == "sets":
        r = r.reshape(len(r), -1).astype(np.int64)
        lost = np.where(r >= 0, flows[np.maximum(r, 0)], 0.0).sum(axis=1)
    elif kind == "elements":
        r = r.reshape(len(r), 2).astype(np.int64)
        lost = np.zeros(len(r))
        base = float(model.base_mva)
        for j, (k, i) in enumerate(r):
            if k == 0:
                lost[j] = flows[i]
            elif k == 1:
                lost[j] = abs(float(model.pg[i])) / base
            else:
                touch = (model.br_from == i) | (model.br_to == i)
                lost[j] = flows[touch].sum() + abs(float(model.pd[i])) / base
    else:
        raise ValueError(f"unknown outage row kind {kind!r}")
    return np.minimum(ITER_BASE + ITER_PER_PU * lost, float(max_iterations))


def balanced_shards(costs: Sequence[float], world: int) -> list:
    """Deal rows to `world` ranks so that their summed costs are even: longest processing time first (rows by
    cost, highest first, each to the rank with the least cost so far; ties to the rank with fewer rows, then the
    lower rank). Returns, per rank, its row positions in ascending order."""
    c = np.asarray(costs, np.float64)
    order = np.argsort(-c, kind="stable")
    heap = [(0.0, 0, r) for r in range(world)]
    heapq.heapify(heap)
    picks = [[] for _ in range(world)]
    for j in order:
        load, cnt, r = heapq.heappop(heap)
        picks[r].append(int(j))
        heapq.heappush(heap, (load + float(c[j]), cnt + 1, r))
    return [np.array(sorted(p), np.int64) for p in picks]


def merge(parts: list) -> dict:
    """Concatenate per-rank raw screen results (rank order) into one, fixing the violation offsets."""
    out = {k: np.concatenate([p[k] for p in parts]) for k in PER_OUTAGE}
    for k in OPTIONAL:
        if all(k in p for p in parts):
            out[k] = np.concatenate([p[k] for p in parts])
    ptr, kinds, elems, vals = [0], [], [], []
    for p in parts:
        base = ptr[-1]
        ptr.extend((p["viol_ptr"][1:] + base).tolist())
        kinds.append(p["viol_kind"])
        elems.append(p["viol_element"])
        vals.append(p["viol_value"])
    out["viol_ptr"] = np.array(ptr, dtype=np.int32)
    out["viol_kind"] = np.concatenate(kinds).astype(np.int32)
    out["viol_element"] = np.concatenate(elems).astype(np.int32)
    out["viol_value"] = np.concatenate(vals)
    return out


def reorder(merged: dict, rows_of: np.ndarray) -> dict:
    """Put a merged result back in the caller's row order: row j of `merged` is the caller's row rows_of[j]."""
    pos = np.empty(len(rows_of), np.int64)
    pos[rows_of] = np.arange(len(rows_of))
    out = {k: v[pos] for k, v in merged.items() if k not in ("viol_ptr", "viol_kind", "viol_element", "viol_value")}
    ptr = np.asarray(merged["viol_ptr"], np.int64)
    lens = (ptr[1:] - ptr[:-1])[pos]
    new_ptr = np.concatenate([[0], np.cumsum(lens)])
    src = np.repeat(ptr[:-1][pos] - new_ptr[:-1], lens) + np.arange(int(new_ptr[-1]))
    out["viol_ptr"] = new_ptr.astype(np.int32)
    for k in ("viol_kind", "viol_element", "viol_value"):
        out[k] = merged[k][src]
    return out


def screen_sharded(model, branch_idx, screen: Callable, group=None, rank: Optional[int] = None,
                   world: Optional[int] = None, costs: Optional[Sequence[float]] = None) -> dict:
    """Screen this rank's shard with ``screen(model, rows_shard) -> raw dict`` and all-gather the results, in the
    caller's row order.

    Without `costs` the shards are contiguous count splits; with them (one estimate per row, e.g.
    :func:`outage_costs`) they are :func:`balanced_shards`. ``group`` is a torch.distributed process group (None =
    the default group, or no distribution when torch.distributed is not initialised)."""
    import torch.distributed as dist
    idx = np.asarray(branch_idx, dtype=np.int32)
    if world is None:
        world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    if rank is None:
        rank = dist.get_rank(group) if world > 1 else 0
    if costs is not None and len(costs) != len(idx):
        raise ValueError(f"{len(costs)} costs for {len(idx)} outage rows")
    if costs is None or world == 1:
        shards = None
        mine_rows = idx[shard(len(idx), rank, world)]
    else:
        shards = balanced_shards(costs, world)
        mine_rows = idx[shards[rank]]
    # rows: a branch, a set of branches, or an element outage's (kind, index) per outage
    mine = screen(model, mine_rows)
    if world == 1:
        return merge([mine])
    keys = PER_OUTAGE + ("viol_ptr", "viol_kind", "viol_element", "viol_value") + tuple(k for k in OPTIONAL if k in mine)
    part = {k: np.asarray(mine[k]) for k in keys}
    parts = [None] * world
    dist.all_gather_object(parts, part, group=group)
    merged = merge(parts)
    if shards is None:
        return merged
    return reorder(merged, np.concatenate(shards))
