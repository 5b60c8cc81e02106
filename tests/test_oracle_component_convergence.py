"""The oracle against the remaining units of the reference's component
convergence verification (verification/sisl_component_convergence.py):
C-grid diff/avg (unit 2), explicit tendencies (5), the implicit linear
operator (6), semi-Lagrangian advection (7) and flux-form advection (8)
converge at second order on 16^3, 32^3, 64^3 grids (the reference prints
"Expected ~2.00").  Units 1, 3 and 4 are in tests/test_oracle_pins.py.
CPU, float64."""

import pytest

import _components as C


@pytest.mark.parametrize("unit", ["unit2_operators", "units5_7", "unit8_ffsl"])
def test_second_order(unit):
    fn = getattr(C, unit)
    errs = [fn(n) for n in (16, 32, 64)]
    for k, r in C.rates(errs).items():
        assert min(r) >= 1.8, (unit, k, r, [e[k] for e in errs])
