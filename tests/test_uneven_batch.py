"""The uneven multi-grid batch (gs_pf_solve_multi: one persistent launch over grids of different sizes) on a B200,
through the C ABI, against the oracle: identical statuses, converged voltages within 1e-8 pu and angles within
1e-8 rad. A second call reuses the autotuned CTA shape and gives the same results bit for bit (a case's arithmetic
does not depend on which CTA runs it)."""
import numpy as np
import pytest

import oracle
from gridsim_b200 import _abi, synthetic
from gridsim_b200.engine import PowerFlowOptions, UnevenBatch
from tests.conftest import golden_model

pytestmark = pytest.mark.gpu

VM_TOL = 1e-8
VA_TOL_RAD = 1e-8
CASES = 6


@pytest.fixture(scope="module")
def population():
    models = [golden_model("case9")[0], golden_model("case118")[0], synthetic.config_grid(0, 0),
              synthetic.make_grid(600, 825, 72, seed=5), golden_model("case14")[0], synthetic.config_grid(1, 0)]
    scales, outs = [], []
    for k, m in enumerate(models):
        scales.append(synthetic.load_scalings(m, CASES, k))
        cand = synthetic.outage_set(m, None, 0)
        o = np.full(CASES, -1, np.int32)
        o[1::2] = cand[(np.arange(CASES // 2) * 7) % len(cand)]
        outs.append(o)
    return models, scales, outs


def _oracle_case(m, scale, outage, opt):
    mk = m.copy()
    mk.pd = m.pd * scale
    mk.qd = m.qd * scale
    if outage >= 0:
        mk.br_in_service = m.br_in_service.copy()
        mk.br_in_service[outage] = 0
    return oracle.solve(mk, opt)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_uneven_batch_matches_the_oracle(population, precision):
    models, scales, outs = population
    opt = PowerFlowOptions(precision=precision, max_iterations=20)
    batch = UnevenBatch(models)
    try:
        r = batch.solve([CASES] * len(models), scales, outs, opt, keep_states=True)
        assert batch.stats["items"] == CASES * len(models)
        assert batch.stats["threads_per_cta"] in (256, 512, 1024)
        for k, m in enumerate(models):
            for c in range(CASES):
                ref = _oracle_case(m, scales[k][c], int(outs[k][c]), opt.to_c())
                assert r["status"][k][c] == ref["status"], (k, c)
                if ref["status"] == _abi.PF_CONVERGED:
                    assert r["max_mismatch"][k][c] < 1e-8
                    assert np.max(np.abs(r["vm"][k][c] - ref["vm"])) <= VM_TOL, (k, c)
                    assert np.max(np.abs(np.radians(r["va_deg"][k][c] - ref["va_deg"]))) <= VA_TOL_RAD, (k, c)
        again = batch.solve([CASES] * len(models), scales, outs, opt, keep_states=True)
        assert batch.stats["tuned_now"] == 0
        for k in range(len(models)):
            assert np.array_equal(again["status"][k], r["status"][k])
            assert np.array_equal(again["vm"][k], r["vm"][k])
            assert np.array_equal(again["va_deg"][k], r["va_deg"][k])
    finally:
        batch.close()


def test_uneven_batch_counts_may_be_zero(population):
    models, scales, outs = population
    batch = UnevenBatch(models[:3])
    try:
        r = batch.solve([0, 2, 0], [scales[0][:0], scales[1][:2], scales[2][:0]], None,
                        PowerFlowOptions(precision="mixed"), keep_states=True)
        assert [len(s) for s in r["status"]] == [0, 2, 0]
        assert (r["status"][1] == _abi.PF_CONVERGED).all()
    finally:
        batch.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_uneven_batch_under_study_options(population, precision):
    """ContingencyAnalysis.StudyOptions (100 iterations, Q limits, the DC retry): each grid's cases run as one batch
    solve, held to the oracle like the persistent launch."""
    from gridsim_b200.engine import study_options
    from tests.conftest import assert_states_close

    models, scales, outs = population
    opt = study_options(precision)
    batch = UnevenBatch(models)
    try:
        r = batch.solve([CASES] * len(models), scales, outs, opt, keep_states=True)
        assert batch.stats["items"] == CASES * len(models)
        for k, m in enumerate(models):
            for c in range(CASES):
                ref = _oracle_case(m, scales[k][c], int(outs[k][c]), opt.to_c())
                assert r["status"][k][c] == ref["status"], (k, c)
                if ref["status"] == _abi.PF_CONVERGED:
                    assert r["max_mismatch"][k][c] < 1e-8
                    assert_states_close(m, [int(outs[k][c])], r["vm"][k][c], r["va_deg"][k][c], ref["vm"], ref["va_deg"],
                                        VM_TOL, VA_TOL_RAD)
    finally:
        batch.close()
