"""The oracle against the reference's manufactured-tendency verification
(verification/equation_tendency_convergence.py): on 16^3, 32^3 and 64^3
oblique-stereographic grids the five explicit tendencies converge to the
analytic ones at second order.  CPU, float64."""

import pytest

import _manufactured as mm


@pytest.mark.parametrize("faces", ["analytic", "averaged"])
def test_explicit_tendencies_second_order(faces):
    errs = [mm.errors("oracle", n, faces=faces) for n in (16, 32, 64)]
    for k, r in mm.rates(errs).items():
        assert r[-1] >= 1.8, (faces, k, r, [e[k] for e in errs])
