"""Euler3D.core keeps the cores of its own background and only the most
recent few of other backgrounds (a fresh precompute_bg dict per call is a
new background).  CPU: Core is replaced by a stand-in that records builds."""

import torch

from _cases import build, mountain


class _FakeCore:
    built = 0

    def __init__(self, *a, **kw):
        _FakeCore.built += 1
        self.rho_bg = kw.get("rho_bg")


def test_foreign_background_cores_are_bounded(monkeypatch):
    import suetes_b200.euler as E
    monkeypatch.setattr(E, "Core", _FakeCore)
    _FakeCore.built = 0
    g, op, ph = build("cuda", 8, 6, 5, 1000.0, 1000.0, 500.0, h=mountain, device="cpu", dt=10.0)
    own = ph.core(torch.float32)
    assert ph.core(torch.float32) is own and _FakeCore.built == 1
    for n in range(3 * E.BG_CORE_CACHE):
        # the keys core() reads of a precompute_bg dict (its stagger averages need CUDA)
        bg = {"th_v": ph.theta_bg + 0.1 * (n + 1), "pi_bg": ph.pi_bg, "rho": 1.0 + 0.0 * ph.pi_bg}
        c = ph.core(torch.float32, bg=bg)
        assert c.rho_bg is bg["rho"]
        assert ph.core(torch.float32, bg=bg) is c  # a hit while cached
    assert len(ph._bg_cores) == E.BG_CORE_CACHE
    assert _FakeCore.built == 1 + 3 * E.BG_CORE_CACHE
    assert ph.core(torch.float32) is own  # the own background's core survives
