"""The allocation-free mismatch check (gs_pf_mismatch_noalloc), through the C ABI, on a B200.

Who needs it: callers that cannot allocate device memory where they check a state -- a loop whose device
memory all comes from its own pool, or code running while a CUDA stream is captured into a graph, where
cudaMalloc is not allowed. The entry point takes the caller's device arrays and keeps its only scratch in a
static device array. This test hands it the final states of a batch solve and checks its max |mismatch|
against the value the batch solve itself reports for those states (gs_pf_solve_batch), twice in a row, so a
second call sees the shared scratch left by the first. Tolerance: rtol 1e-6, atol 1e-11 pu (the states come
back with angles in degrees; converting them to radians again perturbs the last bits).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-11


def test_noalloc_mismatch_matches_the_batch_solve_twice():
    import torch

    from gridsim_b200 import _abi, synthetic
    from gridsim_b200.engine import PowerFlowOptions, SparseNewtonRaphsonPowerFlow

    m = synthetic.config_grid(0, 0)
    idx = synthetic.outage_set(m, None, 0)[:40].astype(np.int32)
    solver = SparseNewtonRaphsonPowerFlow("fp64")
    # a cap of 2 steps leaves some states short of convergence, so the mismatches span many magnitudes
    ref = solver.solve_batch(m, outage=idx, options=PowerFlowOptions(max_iterations=2), keep_states=True)
    grid = solver.grid_for(m)
    count = idx.shape[0]
    dev = torch.device("cuda:0")
    d_vm = torch.tensor(ref["vm"], dtype=torch.float64, device=dev).contiguous()
    d_va = torch.tensor(np.radians(ref["va_deg"]), dtype=torch.float64, device=dev).contiguous()
    d_out = torch.tensor(idx, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    lib = _abi.load_library()
    for call in range(2):
        d_res = torch.full((count,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = lib.gs_pf_mismatch_noalloc(grid.handle, count, ctypes.c_void_p(d_vm.data_ptr()),
                                        ctypes.c_void_p(d_va.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                        ctypes.c_void_p(d_res.data_ptr()))
        assert rc == _abi.GS_OK, grid.ctx.last_error()
        got = d_res.cpu().numpy()
        assert np.allclose(got, ref["max_mismatch"], rtol=RTOL, atol=ATOL), (call, got, ref["max_mismatch"])
        assert got.max() > 1e-10  # non-trivial states


def test_noalloc_refuses_more_systems_than_its_scratch_holds():
    from gridsim_b200 import _abi, synthetic
    from gridsim_b200.engine import SparseNewtonRaphsonPowerFlow

    m = synthetic.config_grid(0, 0)
    grid = SparseNewtonRaphsonPowerFlow("fp64").grid_for(m)
    lib = _abi.load_library()
    dummy = ctypes.c_void_p(16)
    rc = lib.gs_pf_mismatch_noalloc(grid.handle, 65537, dummy, dummy, None, dummy)
    assert rc == _abi.GS_ERR_CAPACITY
    assert "at most 65536" in grid.ctx.last_error()
