"""Two ranks over gloo on CPU: each screens its shard (with the oracle standing in for the device engine) and
the all-gathered result equals the single-process screen."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import oracle
    from gridsim_b200 import _abi, synthetic
    from gridsim_b200.parallel import screen_sharded
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        m = synthetic.config_grid(0, 0)
        idx = synthetic.outage_set(m, None, 0)[:25]
        o = _abi.default_opts()
        o.max_iterations = 20
        o.warm_start_from_base = 1
        got = screen_sharded(m, idx, lambda mm, ii: oracle.screen(mm, ii, o, threads=1))
        if rank == 0:
            np.savez(out_path, **got)
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
    for k in ("status", "iterations", "viol_ptr", "viol_kind", "viol_element", "viol_value", "max_loading_pct"):
        assert np.array_equal(got[k], whole[k]), k
    del torch
