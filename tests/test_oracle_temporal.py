"""The oracle under the reference's pure temporal self-convergence study
(verification/temporal_core_convergence.py): the 24 s warm bubble at
dt = 2, 1, 0.5, 0.25 s converges at second order in time for both cores
(finest order >= 1.7; the oracle measures 1.8-2.0).  CPU, float64."""

import pytest

import _temporal as tc


@pytest.mark.parametrize("core", ["sisl", "split-explicit"])
def test_temporal_second_order(core):
    sols = [tc.run(core, dt) for dt in (2.0, 1.0, 0.5, 0.25)]
    errs, rates = tc.rates(sols)
    for k, r in rates.items():
        assert r[-1] >= 1.7, (core, k, r, errs[k])
