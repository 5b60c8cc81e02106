"""CPU oracle for the SISL timestep: TEST INFRASTRUCTURE ONLY.

This package is a float64 PyTorch-on-CPU restatement of the reference
Suetes regional-3-D SISL core (``suetes/regional3d/*.py``,
``suetes/shared/transforms.py``) plus the third-party JAX routines that path
calls (``jax.scipy.sparse.linalg.gmres``, ``jax.lax.linalg.tridiagonal_solve``,
``jax.scipy.ndimage.map_coordinates``).  Every function cites the reference
file:line it restates.

It exists to *check* the CUDA implementation in ``suetes_b200``: only the
test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product path never calls into this package.

Pinning: the reference ships no golden vectors.  The oracle is pinned by the
reference's own analytic known-answer tests (ported in
``tests/test_oracle_pins.py``), by scipy cross-checks of the trilinear and
tridiagonal kernels, and by committed seeded fixtures generated from this
package (``tests/golden/make_golden.py``).  JAX itself cannot be imported in
this environment, so GMRES iterate-level behaviour is restated from JAX's
published algorithm and is not pinned against a JAX run.

All tensors are float64 on the CPU; every constructor passes the dtype
explicitly so importing this package never changes torch's global defaults.
"""

import torch

DTYPE = torch.float64
