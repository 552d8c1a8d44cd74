import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the engine through the C ABI")


def golden_model(name):
    import json

    from gridsim_b200.model import GridModel
    with open(os.path.join(GOLDEN, name + ".json")) as fh:
        doc = json.load(fh)
    return GridModel.from_dict(doc["model"]), doc["published"]


@pytest.fixture
def study_opts():
    """ContingencyAnalysis.StudyOptions (ContingencyAnalysis.cs:263-268): 100 iterations, Q limits on, and the
    default DC-angle retry (PowerFlowOptions.cs:121)."""
    from gridsim_b200 import _abi
    o = _abi.default_opts()
    o.max_iterations = 100
    o.enforce_q_limits = 1
    o.retry_from_dc_start = 1
    return o


def assert_states_close(m, removed_branches, gpu_vm, gpu_va_deg, ref_vm, ref_va_deg, vm_tol, va_tol_rad, removed_bus=-1):
    """Voltage magnitudes within vm_tol, angles within va_tol_rad, on the buses of the reduced grid.

    A connected part left with no reference bus by the outage, that still balances (a synchronous condenser or a
    zero-injection pair cut off, for example), has angles fixed only up to a common offset: every offset solves its
    equations, and the reference's linear solver and this engine leave it at different ones. There the angles are
    compared as differences from the part's first bus; everywhere else absolutely."""
    n = m.n_bus
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    gone = set(int(k) for k in removed_branches if k >= 0)
    for k in range(m.n_branch):
        if m.br_in_service[k] and k not in gone:
            a, b = find(int(m.br_from[k])), find(int(m.br_to[k]))
            if a != b:
                parent[a] = b
    root = [find(i) for i in range(n)]
    keep = [i for i in range(n) if i != removed_bus]
    slack_parts = {root[i] for i in keep if m.bus_type[i] == 3}
    import numpy as np
    gv, rv = np.asarray(gpu_vm), np.asarray(ref_vm)
    ga, ra = np.radians(np.asarray(gpu_va_deg)), np.radians(np.asarray(ref_va_deg))
    assert np.max(np.abs(gv[keep] - rv[keep])) <= vm_tol
    first = {}
    for i in keep:
        first.setdefault(root[i], i)
    for i in keep:
        if root[i] in slack_parts:
            assert abs(ga[i] - ra[i]) <= va_tol_rad, i
        else:
            f = first[root[i]]
            assert abs((ga[i] - ga[f]) - (ra[i] - ra[f])) <= va_tol_rad, i
