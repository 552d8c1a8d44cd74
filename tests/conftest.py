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
