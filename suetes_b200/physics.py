"""``PhysicsSuite``: the parameterisation container the SISL step calls.

Mirrors ``suetes/physics/base.py:3-69`` with torch tensors.  Tendency schemes
expose ``get_tendencies(state, bg)`` (or, with ``is_ml_closure``,
``get_tendencies(state, bg, ml_params=...)``) and return a dict of arrays;
update schemes expose ``apply_update(state)`` and return the fields they
replace.  The suite's arithmetic is the user's; the SISL step hands its
tendencies of ``u``, ``v``, ``w`` and ``th_v`` to the fused CUDA step
(``sisl_step_physics``) and runs its updates between the step and ``bc_fn``.
"""

import torch


class PhysicsSuite:
    """Tendency schemes (continuous processes) and update schemes
    (instantaneous adjustments), plus the registered tracer keys."""

    def __init__(self):
        self.tendency_schemes = []
        self.update_schemes = []
        self.tracer_keys = []

    def add_tendency_scheme(self, scheme):
        self.tendency_schemes.append(scheme)

    def add_update_scheme(self, scheme):
        self.update_schemes.append(scheme)

    def register_tracer(self, key):
        if key not in self.tracer_keys:
            self.tracer_keys.append(key)

    def get_explicit_tendencies(self, state, bg, interior_mask=None, ml_params=None):
        """Sum of every scheme's tendencies (base.py:28-61), zero-initialised
        for u, v, w, th_v, other keys added as schemes return them, each
        multiplied by ``interior_mask[key]`` where the mask names it."""
        total = {k: torch.zeros_like(state[k]) for k in ("u", "v", "w", "th_v")}
        for scheme in self.tendency_schemes:
            if getattr(scheme, "is_ml_closure", False):
                tends = scheme.get_tendencies(state, bg, ml_params=ml_params)
            else:
                tends = scheme.get_tendencies(state, bg)
            for k, v in tends.items():
                if k not in total:
                    total[k] = torch.zeros_like(v)
                total[k] = total[k] + v
        if interior_mask is not None:
            for k in total:
                if k in interior_mask:
                    total[k] = total[k] * interior_mask[k]
        return total

    def apply_state_updates(self, state):
        """Update schemes in order, each seeing its predecessors' results
        (base.py:63-69)."""
        out = dict(state)
        for scheme in self.update_schemes:
            out.update(scheme.apply_update(out))
        return out
