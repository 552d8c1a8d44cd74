"""The allocation-free mismatch check (gs_pf_mismatch_noalloc), through the C ABI, on a B200.

Who needs it: callers that must not allocate device memory where they check a state -- a host whose device
memory all comes from its own pool reserved up front, or a latency-bound loop where cudaMalloc / cudaFree may
synchronise the whole device. The entry point takes the caller's device arrays and keeps its only scratch in a
static device array shared by every call.

The test hands it states of a batch solve cut short after two Newton steps (so the mismatches span many
magnitudes) and checks its max |mismatch| against
  * the oracle's mismatch of the same states (the reference's BuildY / BuildBusSpec / ComputeInjections restated
    on the CPU), with the outages given and, in a second pair of calls, with no outage array at all (the intact
    grid), and
  * the max mismatch the existing entry point (gs_pf_solve_batch) reports for those states,
each on two calls in a row, so the second call sees the scratch the first one left. Tolerance: rtol 1e-6, atol
1e-11 pu (the states come back with angles in degrees; turning them into radians again perturbs the last bits).
The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-11


def _call(lib, grid, count, d_vm, d_va, d_out):
    import torch
    d_res = torch.full((count,), -1.0, dtype=torch.float64, device=d_vm.device)
    torch.cuda.synchronize()
    rc = lib.gs_pf_mismatch_noalloc(grid.handle, count, ctypes.c_void_p(d_vm.data_ptr()),
                                    ctypes.c_void_p(d_va.data_ptr()),
                                    None if d_out is None else ctypes.c_void_p(d_out.data_ptr()),
                                    ctypes.c_void_p(d_res.data_ptr()))
    assert rc == 0, grid.ctx.last_error()
    return d_res.cpu().numpy()


def test_noalloc_mismatch_matches_the_oracle_and_the_batch_solve_twice():
    import torch

    import oracle
    from gridsim_b200 import _abi, synthetic
    from gridsim_b200.engine import PowerFlowOptions, SparseNewtonRaphsonPowerFlow

    m = synthetic.config_grid(0, 0)
    idx = synthetic.outage_set(m, None, 0)[:40].astype(np.int32)
    solver = SparseNewtonRaphsonPowerFlow("fp64")
    ref = solver.solve_batch(m, outage=idx, options=PowerFlowOptions(max_iterations=2), keep_states=True)
    grid = solver.grid_for(m)
    count = idx.shape[0]
    va_rad = np.radians(ref["va_deg"])
    dev = torch.device("cuda:0")
    d_vm = torch.tensor(ref["vm"], dtype=torch.float64, device=dev).contiguous()
    d_va = torch.tensor(va_rad, dtype=torch.float64, device=dev).contiguous()
    d_out = torch.tensor(idx, dtype=torch.int32, device=dev)
    lib = _abi.load_library()
    want_out = oracle.max_mismatch(m, ref["vm"], va_rad, idx)
    want_intact = oracle.max_mismatch(m, ref["vm"], va_rad, None)
    assert want_out.max() > 1e-10 and not np.allclose(want_out, want_intact)  # the outages matter here
    for call in range(2):
        got = _call(lib, grid, count, d_vm, d_va, d_out)
        assert np.allclose(got, want_out, rtol=RTOL, atol=ATOL), (call, got, want_out)
        assert np.allclose(got, ref["max_mismatch"], rtol=RTOL, atol=ATOL), (call, got, ref["max_mismatch"])
    for call in range(2):
        got = _call(lib, grid, count, d_vm, d_va, None)
        assert np.allclose(got, want_intact, rtol=RTOL, atol=ATOL), (call, got, want_intact)


def test_noalloc_mismatch_takes_voltage_dependent_loads():
    """With ZIP loads (a load drawn as Pd (Ap V^2 + Bp V + Cp), Qd likewise) the mismatch is taken at each state's
    voltages, as the oracle's and the batch solve's are."""
    import torch

    import oracle
    from gridsim_b200 import _abi, synthetic
    from gridsim_b200.engine import PowerFlowOptions, SparseNewtonRaphsonPowerFlow

    m = synthetic.config_grid(0, 0).copy()
    z = np.tile([0.0, 0.0, 1.0, 0.0, 0.0, 1.0], (m.n_bus, 1))
    z[::3] = [0.3, 0.3, 0.4, 0.2, 0.3, 0.5]
    m.zip = z
    idx = synthetic.outage_set(m, None, 0)[:24].astype(np.int32)
    solver = SparseNewtonRaphsonPowerFlow("fp64")
    ref = solver.solve_batch(m, outage=idx, options=PowerFlowOptions(max_iterations=2), keep_states=True)
    grid = solver.grid_for(m)
    va_rad = np.radians(ref["va_deg"])
    dev = torch.device("cuda:0")
    d_vm = torch.tensor(ref["vm"], dtype=torch.float64, device=dev).contiguous()
    d_va = torch.tensor(va_rad, dtype=torch.float64, device=dev).contiguous()
    d_out = torch.tensor(idx, dtype=torch.int32, device=dev)
    want = oracle.max_mismatch(m, ref["vm"], va_rad, idx)
    lib = _abi.load_library()
    for call in range(2):
        got = _call(lib, grid, idx.shape[0], d_vm, d_va, d_out)
        assert np.allclose(got, want, rtol=RTOL, atol=ATOL), (call, got, want)
        assert np.allclose(got, ref["max_mismatch"], rtol=RTOL, atol=ATOL), (call, got, ref["max_mismatch"])


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
