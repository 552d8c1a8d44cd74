"""Two ranks over gloo on CPU: each screens its shard (with the oracle standing in for the device engine) and
the all-gathered result equals the single-process screen, for contiguous and for cost-balanced shards."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pairs(m):
    """21 two-branch outages of the 120-bus grid, bridges among them (some split the grid)."""
    from gridsim_b200 import synthetic
    live = m.in_service_branches()
    br = np.nonzero(synthetic.bridges(m))[0][:3]
    rows = [[int(live[3 * k]), int(live[3 * k + 1])] for k in range(18)] + [[int(b), int(live[0])] for b in br]
    return np.array(rows, np.int32)


def _elements(m):
    """(kind, index) rows: every in-service generator, then the first 15 buses."""
    on = np.nonzero(m.gen_in_service)[0]
    return np.array([[1, int(g)] for g in on] + [[2, i] for i in range(15)], np.int32)


def _shared(m, rows):
    """The element screen with governor-droop sharing; its notes under the engine's key."""
    import oracle
    from gridsim_b200 import _abi
    o = _abi.default_opts()
    o.max_iterations = 20
    r = oracle.screen_elements(m, rows[:, 0], rows[:, 1], o, threads=1, dispatch="droop")
    r["share_notes"] = r.pop("notes")
    return r


def _worker(rank, world, port, out_path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import oracle
    from gridsim_b200 import _abi, synthetic
    from gridsim_b200.parallel import outage_costs, screen_sharded
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = synthetic.config_grid(0, 0)
        idx = synthetic.outage_set(m, None, 0)[:25]
        o = _abi.default_opts()
        o.max_iterations = 20
        o.warm_start_from_base = 1
        got = screen_sharded(m, idx, lambda mm, ii: oracle.screen(mm, ii, o, threads=1))
        pairs = _pairs(m)
        got2 = screen_sharded(m, pairs, lambda mm, ss: oracle.screen_sets(mm, ss, o, threads=1))
        got3 = screen_sharded(m, _elements(m), lambda mm, ee: _shared(mm, ee))
        # cost-balanced shards (rows dealt by estimated iterations), merged back in the caller's row order
        got4 = screen_sharded(m, idx, lambda mm, ii: oracle.screen(mm, ii, o, threads=1), costs=outage_costs(m, idx))
        got5 = screen_sharded(m, pairs, lambda mm, ss: oracle.screen_sets(mm, ss, o, threads=1),
                              costs=outage_costs(m, pairs, "sets"))
        els = _elements(m)
        got6 = screen_sharded(m, els, lambda mm, ee: _shared(mm, ee), costs=outage_costs(m, els, "elements"))
        if rank == 0:
            np.savez(out_path, **got)
            np.savez(out_path + ".pairs.npz", **got2)
            np.savez(out_path + ".elements.npz", **got3)
            np.savez(out_path + ".balanced.npz", **got4)
            np.savez(out_path + ".balanced_pairs.npz", **got5)
            np.savez(out_path + ".balanced_elements.npz", **got6)
    finally:
        dist.destroy_process_group()


def test_two_rank_screen_equals_one_process(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    import oracle
    from gridsim_b200 import _abi, synthetic
    out = str(tmp_path / "merged.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    got = np.load(out)
    m = synthetic.config_grid(0, 0)
    idx = synthetic.outage_set(m, None, 0)[:25]
    o = _abi.default_opts()
    o.max_iterations = 20
    o.warm_start_from_base = 1
    whole = oracle.screen(m, idx, o)
    for k in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element", "viol_value", "max_loading_pct",
              "islanded", "worst_boundary_pct"):
        assert np.array_equal(got[k], whole[k]), k
    # multi-branch outages shard by rows the same way
    got2 = np.load(out + ".pairs.npz")
    whole2 = oracle.screen_sets(m, _pairs(m), o)
    for k in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element", "islanded"):
        assert np.array_equal(got2[k], whole2[k]), k
    # element outages with shared dispatch shard by (kind, index) rows, their notes gathered in order
    got3 = np.load(out + ".elements.npz", allow_pickle=True)
    whole3 = _shared(m, _elements(m))
    for k in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element", "islanded"):
        assert np.array_equal(got3[k], whole3[k]), k
    assert list(got3["share_notes"]) == list(whole3["share_notes"])
    assert any(n is not None for n in whole3["share_notes"])
    # the cost-balanced shards give the same screens, row for row
    for suffix, ref in ((".balanced.npz", whole), (".balanced_pairs.npz", whole2), (".balanced_elements.npz", whole3)):
        got_b = np.load(out + suffix, allow_pickle=True)
        for k in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element", "viol_value", "islanded"):
            assert np.array_equal(got_b[k], ref[k]), (suffix, k)
    assert list(np.load(out + ".balanced_elements.npz", allow_pickle=True)["share_notes"]) == list(whole3["share_notes"])
    del torch
