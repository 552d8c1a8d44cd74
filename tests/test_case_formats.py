"""The case formats' ratings, boundaries and machine data (CPU): MATPOWER RATE_B / RATE_C read as the reference reads them
(tests/GridSim.Tests/ContingencyTypesAndRatingsTests.cs:43-51, case24_ieee_rts), the JSON case directory's
ratingBMva / ratingCMva multiplied by `circuits` like ratingMva (:75-96), the units' machine data of both formats,
and a round trip of names, ratings, transformers, boundaries and machine data through the JSON writer and reader."""
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


def test_matpower_machine_data_is_read():
    """PMIN / PMAX / MBASE of mpc.gen (MatpowerParser.cs:272-307): case9's units are rated 250, 300 and 270 MW on a
    100 MVA machine base, with H 0 (MATPOWER carries no inertia)."""
    m, _ = golden_model("case9")
    assert list(m.pmax) == [250.0, 300.0, 270.0]
    assert list(m.pmin) == [10.0, 10.0, 10.0]
    assert list(m.mbase) == [100.0, 100.0, 100.0]
    assert not m.inertia_h.any()


def test_json_machine_data_defaults_and_round_trip(tmp_path):
    """JsonGridLoader.cs:158-170: Pmin 0 and Pmax capacityMva unless written, MBase capacityMva, H inertiaH, the
    type "ccgt" unless written; the writer keeps every field."""
    d = tmp_path / "case"
    d.mkdir()
    files = {
        "system.json": {"name": "t", "baseMva": 100, "frequencyHz": 50, "dispatch": False},
        "buses.json": [{"id": 1, "baseKv": 132, "type": "slack"}, {"id": 2, "baseKv": 132}],
        "generation.json": [{"name": "G", "bus": 1, "capacityMva": 120, "outputMw": 10, "role": "slack"},
                            {"name": "W", "bus": 2, "capacityMva": 80, "outputMw": 5, "pMinMw": 1, "pMaxMw": 60,
                             "inertiaH": 0.5, "type": "wind_offshore", "converterInterfaced": True},
                            {"name": "S", "bus": 2, "capacityMva": 30, "outputMw": 0, "powerFlowOnly": True}],
        "demand.json": [{"bus": 2, "pMw": 15}],
        "transmission.json": [{"name": "L", "from": 1, "to": 2, "rPu": 0.01, "xPu": 0.1, "ratingMva": 50}],
    }
    for name, obj in files.items():
        (d / name).write_text(json.dumps(obj))
    m = load_case_dir(str(d))
    assert list(m.pmin) == [0.0, 1.0, 0.0] and list(m.pmax) == [120.0, 60.0, 30.0]
    assert list(m.mbase) == [120.0, 80.0, 30.0] and list(m.inertia_h) == [0.0, 0.5, 0.0]
    assert m.gen_type == ["ccgt", "wind_offshore", "ccgt"]
    assert list(m.pf_only) == [0, 0, 1] and list(m.converter) == [-1, 1, -1]
    out = tmp_path / "again"
    save_case_dir(m, str(out))
    m2 = load_case_dir(str(out))
    for key in ("pmin", "pmax", "mbase", "inertia_h", "pf_only", "converter", "pg", "qmin", "qmax"):
        assert np.array_equal(getattr(m, key), getattr(m2, key)), key
    assert m2.gen_type == m.gen_type
