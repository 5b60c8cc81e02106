"""``Simulation``: the chunked time-integration driver.

Mirrors ``suetes/shared/driver.py:7-132``.  ``run`` advances a state with
``step_fn(state, step_idx) -> (state, metrics)`` in chunks of
``chunk_steps``, reporting the largest ``|metrics|`` (max |w| in the
reference's runs) per chunk; the device work of a chunk is queued without
host synchronisation until the chunk ends (the reference's jitted
``lax.scan`` per chunk).  ``run_differentiable`` is the autograd form with
``step_fn(state, t, forcing=..., bc_fn=...)``: each chunk is recomputed in
the backward pass instead of storing its intermediate states
(``jax.checkpoint`` around the chunk scan in the reference).
"""

import time

import torch
from torch.utils.checkpoint import checkpoint


def _sync(state):
    for v in state.values() if isinstance(state, dict) else ():
        if torch.is_tensor(v) and v.is_cuda:
            torch.cuda.synchronize(v.device)
            return


class Simulation:
    """Manages the time-integration loop and its chunking."""

    def __init__(self, step_fn, dt):
        self.step_fn = step_fn
        self.dt = dt

    def run(self, initial_state, t_start, t_end, chunk_steps=120, log=print):
        total = int((t_end - t_start) / self.dt)
        n_chunks, remainder = divmod(total, chunk_steps)
        log(f"[SIMULATION] Starting: T={t_start} -> T={t_end}")
        log(f"[SIMULATION] Total Steps: {total}")
        log(f"[SIMULATION] Chunk Size:  {chunk_steps} steps")
        state = initial_state
        step = int(t_start / self.dt)
        start = time.time()

        def chunk(state, step, n):
            peak = None
            for off in range(n):
                state, metrics = self.step_fn(state, step + off)
                if metrics is not None:
                    m = torch.as_tensor(metrics).abs().max()
                    peak = m if peak is None else torch.maximum(peak, m.to(peak.device))
            _sync(state)
            return state, (float(peak) if peak is not None else 0.0)

        for _ in range(n_chunks):
            t0 = time.time()
            state, peak = chunk(state, step, chunk_steps)
            step += chunk_steps
            log(f"    Progress: {step * self.dt:.1f}s / {t_end:.1f}s | Max W: {peak:.4f} m/s | "
                f"Chunk Wall Time: {time.time() - t0:.2f}s")
        if remainder:
            log(f"    Finishing remaining {remainder} steps...")
            state, _ = chunk(state, step, remainder)
        log(f"[Simulation] Done in {time.time() - start:.2f}s\n")
        return state

    def run_differentiable(self, initial_state, t_start, t_end, bc_fn=None, forcing=None, chunk_steps=50):
        """The integration as an autograd graph whose chunks are recomputed in
        the backward pass (driver.py:91-132)."""
        total = int((t_end - t_start) / self.dt)
        n_chunks, remainder = divmod(total, chunk_steps)
        start = int(t_start / self.dt)

        def steps(state, first, n):
            for off in range(n):
                state = self.step_fn(state, (first + off) * self.dt, forcing=forcing, bc_fn=bc_fn)
            return state

        state = initial_state
        for c in range(n_chunks):
            keys = [k for k, v in state.items() if torch.is_tensor(v)]
            rest = {k: v for k, v in state.items() if not torch.is_tensor(v)}
            side = {}

            def run_chunk(*tensors, keys=keys, rest=rest, side=side, first=start + c * chunk_steps):
                out = steps({**rest, **dict(zip(keys, tensors))}, first, chunk_steps)
                side["keys"] = [k for k, v in out.items() if torch.is_tensor(v)]
                side["rest"] = {k: v for k, v in out.items() if not torch.is_tensor(v)}
                return tuple(out[k] for k in side["keys"])

            outs = checkpoint(run_chunk, *[state[k] for k in keys], use_reentrant=False)
            state = {**side["rest"], **dict(zip(side["keys"], outs))}
        if remainder:
            state = steps(state, start + n_chunks * chunk_steps, remainder)
        return state
