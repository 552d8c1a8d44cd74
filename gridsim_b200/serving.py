"""The request loop over the gridsim_b200 C ABI (``gs_serve_*``): load-flow requests on grids kept resident on the
GPU, stepped by continuous batching.

The reference's nearest counterpart is its sequential ``gridsim rpc`` host
(``src/GridSim.Cli/RpcCommand.cs:11-50``), which runs one ``solve`` at a time. Here every registered grid keeps
its symbolic data, solved base case and a batch of request slots on the device; a native scheduler thread steps
the occupied slots of each grid one Newton iteration at a time on the grid's own stream, admits queued requests
into slots as they free up, and answers each request as soon as its system stops. A request is a base case
(``outage=-1``) or one branch outage of a registered grid; its result does not depend on what else is in flight.

    server = LoadFlowServer(PowerFlowOptions(precision="mixed", max_iterations=20, warm_start_from_base=True))
    g = server.add_grid(model)
    server.start()
    tickets = server.submit([(g, -1), (g, 17, True)])
    responses = server.poll(timeout_ms=1000)
    server.close()
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Iterable, List, Optional

import numpy as np

from . import _abi
from .engine import CudaContext, CudaGrid, EngineError, PowerFlowOptions
from .model import GridModel

# numpy view of gs_request, so that large submissions need no Python loop
REQUEST_DTYPE = np.dtype([("grid", "<i4"), ("outage", "<i4"), ("want_state", "<i4"), ("reserved", "<i4"),
                          ("tag", "<u8")])
assert REQUEST_DTYPE.itemsize == ctypes.sizeof(_abi.Request)


@dataclass
class ServeResponse:
    ticket: int
    tag: int
    grid: int
    outage: int
    status: int
    iterations: int
    max_mismatch: float
    queue_ms: float
    latency_ms: float
    vm: Optional[np.ndarray] = None       # pu, when the request asked for its state
    va_deg: Optional[np.ndarray] = None

    @property
    def status_name(self) -> str:
        return _abi.PF_STATUS_NAMES[self.status]

    @property
    def converged(self) -> bool:
        return self.status == _abi.PF_CONVERGED


class LoadFlowServer:
    """gs_server: register grids, start, then submit and poll from any thread. With Q limits or the DC retry in
    the options (the reference's rpc solve runs with Q limits, ``src/GridSim.Cli/RpcCommand.cs:675-676``) the loop
    answers each grid's queued requests in batches; warm starts are refused then, and no other solve may use the
    context while the loop runs."""

    def __init__(self, options: Optional[PowerFlowOptions] = None, ctx: Optional[CudaContext] = None,
                 slots_per_grid: int = 0, state_slots: int = 0, hbm_fraction: float = 0.0, scheduler_threads: int = 0):
        self.ctx = ctx or CudaContext.default()
        self.lib = self.ctx.lib
        self.options = options or PowerFlowOptions()
        o = _abi.ServeOpts()
        o.pf = self.options.device_c()
        o.slots_per_grid = slots_per_grid
        o.state_slots = state_slots
        o.hbm_fraction = hbm_fraction
        o.scheduler_threads = scheduler_threads
        self.handle = ctypes.c_void_p()
        self.ctx.check(self.lib.gs_serve_create(self.ctx.handle, ctypes.byref(o), ctypes.byref(self.handle)),
                       "gs_serve_create")
        self.grids: List[CudaGrid] = []
        self._n_bus: List[int] = []
        self._resp = (_abi.Response * 4096)()
        self._state = np.zeros(0)

    def add_grid(self, model: GridModel) -> int:
        g = CudaGrid(self.options.device_model(model), self.ctx)
        idx = ctypes.c_int32()
        self.ctx.check(self.lib.gs_serve_add_grid(self.handle, g.handle, ctypes.byref(idx)), "gs_serve_add_grid")
        self.grids.append(g)
        self._n_bus.append(model.n_bus)
        return idx.value

    def start(self) -> None:
        self.ctx.check(self.lib.gs_serve_start(self.handle), "gs_serve_start")
        self._state = np.zeros(2 * max(self._n_bus) * 64)

    def submit(self, requests) -> np.ndarray:
        """Queue requests: a REQUEST_DTYPE array, or an iterable of (grid, outage[, want_state[, tag]]).
        Returns their tickets."""
        if isinstance(requests, np.ndarray) and requests.dtype == REQUEST_DTYPE:
            arr = np.ascontiguousarray(requests)
        else:
            rows = [tuple(r) for r in requests]
            arr = np.zeros(len(rows), REQUEST_DTYPE)
            for k, r in enumerate(rows):
                arr[k]["grid"], arr[k]["outage"] = r[0], r[1]
                arr[k]["want_state"] = int(r[2]) if len(r) > 2 else 0
                arr[k]["tag"] = int(r[3]) if len(r) > 3 else 0
        tickets = np.zeros(len(arr), np.uint64)
        if len(arr):
            self.ctx.check(self.lib.gs_serve_submit(self.handle, len(arr), arr.ctypes.data_as(ctypes.c_void_p),
                                                    tickets.ctypes.data_as(ctypes.c_void_p)), "gs_serve_submit")
        return tickets

    def poll(self, max_responses: int = 4096, timeout_ms: int = 0) -> List[ServeResponse]:
        """Finished requests (at most max_responses), waiting up to timeout_ms for the first."""
        got = ctypes.c_int32()
        k = min(max_responses, len(self._resp))
        self.ctx.check(self.lib.gs_serve_poll(self.handle, k, timeout_ms, self._resp,
                                              self._state.ctypes.data_as(ctypes.c_void_p), len(self._state),
                                              ctypes.byref(got)), "gs_serve_poll")
        out = []
        for j in range(got.value):
            r = self._resp[j]
            resp = ServeResponse(int(r.ticket), int(r.tag), r.grid, r.outage, r.status, r.iterations, r.max_mismatch,
                                 r.queue_ms, r.latency_ms)
            if r.state_offset >= 0:
                n = self._n_bus[r.grid]
                s = self._state[r.state_offset:r.state_offset + 2 * n]
                resp.vm, resp.va_deg = s[:n].copy(), s[n:].copy()
            out.append(resp)
        return out

    def stats(self) -> dict:
        st = _abi.ServeStats()
        self.ctx.check(self.lib.gs_serve_stats_get(self.handle, ctypes.byref(st)), "gs_serve_stats_get")
        return {f: getattr(st, f) for f, _ in _abi.ServeStats._fields_ if f != "reserved"}

    def stop(self, timeout_ms: int = 60000) -> None:
        if self.handle:
            self.ctx.check(self.lib.gs_serve_stop(self.handle, timeout_ms), "gs_serve_stop")

    def close(self) -> None:
        if self.handle:
            self.lib.gs_serve_destroy(self.handle)
            self.handle = ctypes.c_void_p()
        for g in self.grids:
            g.close()
        self.grids = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def drain(server: LoadFlowServer, count: int, timeout_s: float = 120.0) -> List[ServeResponse]:
    """Poll until `count` responses have arrived (EngineError if they do not within timeout_s)."""
    import time
    out: List[ServeResponse] = []
    t_end = time.monotonic() + timeout_s
    while len(out) < count:
        if time.monotonic() > t_end:
            raise EngineError(f"{count - len(out)} of {count} requests unanswered after {timeout_s} s")
        out.extend(server.poll(timeout_ms=50))
    return out
