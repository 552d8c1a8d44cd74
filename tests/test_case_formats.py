"""The case formats' ratings and boundaries (CPU): MATPOWER RATE_B / RATE_C read as the reference reads them
(tests/GridSim.Tests/ContingencyTypesAndRatingsTests.cs:43-51, case24_ieee_rts), the JSON case directory's
ratingBMva / ratingCMva multiplied by `circuits` like ratingMva (:75-96), and a round trip of names, ratings,
transformers and boundaries through the JSON writer and reader."""
import json
import os

import numpy as np
import pytest

from gridsim_b200 import synthetic
from gridsim_b200.model import load_case_dir, save_case_dir
from tests.conftest import golden_model


def test_matpower_rate_b_and_c_are_read():
    m, _ = golden_model("case24_ieee_rts")
    assert (m.rate_a[0], m.rate_b[0], m.rate_c[0]) == (175.0, 250.0, 200.0)  # branch 1-2
    assert (m.rate_b[1], m.rate_c[1]) == (208.0, 220.0)


def test_json_rating_b_and_c_are_per_circuit(tmp_path):
    d = tmp_path / "case"
    d.mkdir()
    files = {
        "system.json": {"name": "t", "baseMva": 100, "frequencyHz": 50, "dispatch": False},
        "buses.json": [{"id": 1, "baseKv": 132, "type": "slack"}, {"id": 2, "baseKv": 132}],
        "generation.json": [{"name": "G", "bus": 1, "capacityMva": 100, "outputMw": 10, "role": "slack"}],
        "demand.json": [{"bus": 2, "pMw": 10}],
        "transmission.json": [{"name": "L", "from": 1, "to": 2, "rPu": 0.01, "xPu": 0.1, "ratingMva": 50,
                               "ratingBMva": 60, "ratingCMva": 70, "circuits": 2}],
    }
    for fn, obj in files.items():
        (d / fn).write_text(json.dumps(obj))
    m = load_case_dir(str(d))
    assert (m.rate_a[0], m.rate_b[0], m.rate_c[0]) == (100.0, 120.0, 140.0)


def test_json_round_trip_of_names_ratings_and_boundaries(tmp_path):
    m = synthetic.config_grid(0, 0)
    m.br_name = [f"L{k}" for k in range(m.n_branch)]
    m.rate_b = np.where(np.arange(m.n_branch) % 3 == 0, 1.5 * m.rate_a, 0.0)
    m.rate_c = 2.0 * m.rate_a
    m.boundaries = [("north", 120.0, [("L1", 1), ("L4", -1)]), ("none", 0.0, [("L7", 1)])]
    save_case_dir(m, str(tmp_path / "c"))
    back = load_case_dir(str(tmp_path / "c"))
    assert back.br_name == m.br_name
    assert np.allclose(back.rate_b, m.rate_b) and np.allclose(back.rate_c, m.rate_c)
    assert back.boundaries == m.boundaries
    ptr, br, dr, lim = back.boundary_members()
    assert ptr.tolist() == [0, 2, 3] and br.tolist() == [1, 4, 7] and dr.tolist() == [1, -1, 1]
    assert lim.tolist() == [120.0, 0.0]


def test_json_transformers_follow_the_lines(tmp_path):
    d = tmp_path / "case"
    d.mkdir()
    files = {
        "system.json": {"name": "t", "baseMva": 100, "dispatch": False},
        "buses.json": [{"id": 1, "baseKv": 132, "type": "slack"}, {"id": 2, "baseKv": 132}, {"id": 3, "baseKv": 33}],
        "generation.json": [{"name": "G", "bus": 1, "capacityMva": 100, "outputMw": 10, "role": "slack"}],
        "demand.json": [{"bus": 3, "pMw": 10}],
        "transmission.json": [{"name": "L", "from": 1, "to": 2, "rPu": 0.01, "xPu": 0.1, "bPu": 0.02,
                               "ratingMva": 50}],
        "transformer.json": [{"name": "T", "from": 2, "to": 3, "rPu": 0.002, "xPu": 0.08, "tapRatio": 1.02,
                              "ratingMva": 40, "ratingBMva": 45}],
    }
    for fn, obj in files.items():
        (d / fn).write_text(json.dumps(obj))
    m = load_case_dir(str(d))
    assert m.n_branch == 2 and m.br_name == ["L", "T"]
    assert m.is_transformer.tolist() == [0, 1] and m.b[1] == 0.0 and m.tap[1] == 1.02
    assert (m.rate_a[1], m.rate_b[1], m.rate_c[1]) == (40.0, 45.0, 0.0)
