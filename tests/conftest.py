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


# A part without a reference bus is solved, as in the reference, through the singular-step fallback (ILU(0) +
# BiCGSTAB): its common angle offset comes from the iteration's rounding, amplified along the null space. With the
# engine running that fallback in the reference's order and roundings, the offsets agree within 2.1e-8 rad on every
# such outage of the tests; the bound below holds them to that, beside the 1e-8 bar on the in-part differences.
FLOATING_PART_ABS_TOL_RAD = 1e-7


def assert_states_close(m, removed_branches, gpu_vm, gpu_va_deg, ref_vm, ref_va_deg, vm_tol, va_tol_rad, removed_bus=-1):
    """Voltage magnitudes within vm_tol, angles within va_tol_rad, on the buses of the reduced grid.

    A connected part left with no reference bus by the outage, that still balances (a synchronous condenser or a
    zero-injection pair cut off, for example), has angles fixed only up to a common offset: every offset solves its
    equations, and the reference's linear solver and this engine leave it at different ones. There the angles are
    compared as differences from the part's first bus (and absolutely within FLOATING_PART_ABS_TOL_RAD); everywhere
    else absolutely."""
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
            assert abs(ga[i] - ra[i]) <= va_tol_rad, (i, ga[i] - ra[i])
        else:
            f = first[root[i]]
            assert abs((ga[i] - ga[f]) - (ra[i] - ra[f])) <= va_tol_rad, i
            assert abs(ga[i] - ra[i]) <= FLOATING_PART_ABS_TOL_RAD, (i, ga[i] - ra[i])


def resistive_leaf_grid(at_bus: int = 4, r: float = 0.05):
    """case9 with a tenth bus hung from bus `at_bus` (position) by a purely resistive branch (x = 0), carrying 10 MW
    and 3 MVAr of load, every PQ bus starting at 1 pu and 0 degrees and the new bus at its neighbour's start.

    At that start the new bus's 2 x 2 Jacobian block is [[0, N], [M, 0]]: with no reactance between equal voltages
    dP/dtheta and dQ/dV vanish, so a diagonal pivot of a leaf bus (eliminated before its neighbour) collapses in any
    order, while the matrix is regular and the reference's row partial pivoting takes the off-diagonal entries."""
    import numpy as np
    m, _ = golden_model("case9")
    m = m.copy()
    n = m.n_bus

    def app(name, v):
        a = getattr(m, name)
        if a is not None:
            setattr(m, name, np.concatenate([a, np.array([v], dtype=a.dtype)]))
    for name, v in (("bus_id", int(m.bus_id.max()) + 1), ("bus_type", 1), ("pd", 10.0), ("qd", 3.0), ("gs", 0.0),
                    ("bs", 0.0), ("vm", 1.0), ("va_deg", 0.0), ("vmin", np.nan), ("vmax", np.nan),
                    ("base_kv", float(m.base_kv[at_bus]))):
        app(name, v)
    if m.zip is not None:
        m.zip = np.vstack([m.zip, [0.0, 0.0, 1.0, 0.0, 0.0, 1.0]])
    for name, v in (("br_from", at_bus), ("br_to", n), ("r", r), ("x", 0.0), ("b", 0.0), ("tap", 0.0),
                    ("shift_deg", 0.0), ("rate_a", 0.0), ("br_in_service", 1), ("is_transformer", 0), ("rate_b", 0.0),
                    ("rate_c", 0.0)):
        app(name, v)
    if m.br_name is not None:
        m.br_name = list(m.br_name) + [""]
    m.vm[:] = np.where(m.bus_type == 1, 1.0, m.vm)
    m.va_deg[:] = 0.0
    m.vm[n] = m.vm[at_bus]
    return m
