"""The reference's manufactured-tendency verification
(verification/equation_tendency_convergence.py) on the CUDA explicit
kernel, float64: second-order convergence of the five explicit tendencies on
16^3, 32^3 and 64^3 oblique-stereographic grids, every error within 1e-6
(relative) of the oracle's given the same face averages of theta'."""

import pytest

import _manufactured as mm

pytestmark = pytest.mark.gpu


def test_explicit_tendencies_second_order():
    errs = [mm.errors("cuda", n, device="cuda") for n in (16, 32, 64)]
    for k, r in mm.rates(errs).items():
        assert r[-1] >= 1.8, (k, r, [e[k] for e in errs])
    ref = [mm.errors("oracle", n, faces="averaged") for n in (16, 32, 64)]
    for e, o in zip(errs, ref):
        for k in e:
            assert abs(e[k] - o[k]) <= 1e-6 * o[k], (k, e[k], o[k])
