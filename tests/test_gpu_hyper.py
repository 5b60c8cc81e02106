"""``Euler3D.diffusion`` (HyperFilter, diffusion.py:80-173) on the CUDA
kernels against the float64 oracle's filter."""

import pytest
import torch

from _cases import build, mountain, rel_l2, to_cuda

pytestmark = pytest.mark.gpu


def test_hyperfilter_matches_oracle():
    kw = dict(dt=10.0, N_bv=0.01, nu_h_factor=0.05, nu_div_factor=0.1)
    o = build("oracle", 14, 12, 10, 500.0, 500.0, 500.0, h=mountain, **kw)
    p = build("cuda", 14, 12, 10, 500.0, 500.0, 500.0, h=mountain, device="cuda", **kw)
    g = torch.Generator().manual_seed(9)
    r = lambda *s: torch.randn(*s, generator=g, dtype=torch.float64)
    sp = {"u": r(15, 12, 10), "v": r(14, 13, 10), "w": 0.1 * r(14, 12, 11), "th_v": o[2].theta_bg + r(14, 12, 10)}
    bo = o[2].precompute_bg(o[2].bg_state_ref())
    ref = o[2].diffusion.get_tendencies(sp, bo)
    bp = p[2].precompute_bg(p[2].bg_state_ref())
    out = p[2].diffusion.get_tendencies(to_cuda(sp), bp)
    assert set(out) == set(ref) == {"u", "v", "w", "th_v"}
    for k in ref:
        assert rel_l2(out[k], ref[k]) < 1e-11, (k, rel_l2(out[k], ref[k]))
