"""Sharding the N-1 screen over ranks (one process per GPU).

The outages of a screen are independent, so they are split into contiguous, balanced shards, each rank screens
its shard on its own GPU, and the per-outage results are gathered in rank order (an all-gather of the compact
result records, a few tens of bytes per outage plus the violation list; no collective runs on the data path).
The reference screens outages with a thread pool instead (ContingencyAnalysis.ScreenBranchesParallel,
``src/GridSim.Core/Analysis/ContingencyAnalysis.cs:323-344``); results come back in branch order either way.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

PER_OUTAGE = ("status", "iterations", "max_mismatch", "min_vm", "max_vm", "max_loading_pct")
OPTIONAL = ("worst_boundary_pct", "islanded", "share_notes")  # merged when every part has them


def shard(n_items: int, rank: int, world: int) -> slice:
    """Contiguous balanced split: the first n % world ranks get one item more."""
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


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


def screen_sharded(model, branch_idx, screen: Callable, group=None, rank: Optional[int] = None,
                   world: Optional[int] = None) -> dict:
    """Screen this rank's shard with ``screen(model, idx_shard) -> raw dict`` and all-gather the results.

    ``group`` is a torch.distributed process group (None = the default group, or no distribution when
    torch.distributed is not initialised)."""
    import torch.distributed as dist
    idx = np.asarray(branch_idx, dtype=np.int32)
    if world is None:
        world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    if rank is None:
        rank = dist.get_rank(group) if world > 1 else 0
    # rows: a branch, a set of branches, or an element outage's (kind, index) per outage
    mine = screen(model, idx[shard(len(idx), rank, world)])
    if world == 1:
        return merge([mine])
    keys = PER_OUTAGE + ("viol_ptr", "viol_kind", "viol_element", "viol_value") + tuple(k for k in OPTIONAL if k in mine)
    part = {k: np.asarray(mine[k]) for k in keys}
    parts = [None] * world
    dist.all_gather_object(parts, part, group=group)
    return merge(parts)
