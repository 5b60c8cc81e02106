"""The oracle against the reference's smooth-mode verification gate
(verification/smooth_mode_core_convergence.py): standing gravity and
acoustic modes converge at order >= 1.7 under timestep halving for the SISL
and split-explicit cores.  CPU, float64."""

import pytest

import _smooth_modes as sm


@pytest.mark.parametrize("core", ["sisl", "split-explicit"])
@pytest.mark.parametrize("case", ["gravity", "acoustic"])
def test_smooth_mode_order(case, core):
    cfg = sm.CASES[case]
    sols = [sm.run("oracle", case, core, dt) for dt in cfg["dt"]]
    errs, rates = sm.orders(sols, cfg["fields"])
    for f, r in rates.items():
        assert r[-1] >= sm.WAVE_ORDER, (case, core, f, r, errs[f])
        assert errs[f][-1] < errs[f][0], (case, core, f, errs[f])
