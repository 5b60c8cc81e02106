"""The reference's smooth-mode verification gate
(verification/smooth_mode_core_convergence.py) on the CUDA cores, float64:
standing gravity and acoustic modes converge at order >= 1.7 under
timestep halving, and every self-convergence error is the oracle's
(tests/test_oracle_smooth_modes.py) to within 2 %."""

import pytest

import _smooth_modes as sm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("core", ["sisl", "split-explicit"])
@pytest.mark.parametrize("case", ["gravity", "acoustic"])
def test_smooth_mode_order(case, core):
    cfg = sm.CASES[case]
    sols = [sm.run("cuda", case, core, dt, device="cuda") for dt in cfg["dt"]]
    errs, rates = sm.orders(sols, cfg["fields"])
    for f, r in rates.items():
        assert r[-1] >= sm.WAVE_ORDER, (case, core, f, r, errs[f])
    # the coarsest pair against the oracle's (the finer ones cost the CPU minutes)
    ref = [sm.run("oracle", case, core, dt) for dt in cfg["dt"][:2]]
    rerr, _ = sm.orders(ref, cfg["fields"])
    for f in cfg["fields"]:
        assert abs(errs[f][0] - rerr[f][0]) <= 0.02 * rerr[f][0], (case, core, f, errs[f][0], rerr[f][0])
        assert sm._cropped(sols[0][f]).shape == sm._cropped(ref[0][f]).shape
