"""The allocation-free line transport (sisl_ffsl_lines_noalloc).

Callers that cannot call cudaMalloc while they run -- a stream being
captured into a CUDA graph in global mode, a host model that only lends the
library buffers it pre-sized from its own pool, an FFI handler registered
without a workspace -- use this entry point: its float64 scratch is a fixed
8 MiB device array instead of a caller workspace.  The test calls it through
the C ABI twice in a row, with different inputs, and checks each result
against the workspace-taking sisl_ffsl_lines on the same inputs; it also
checks that a problem larger than the fixed scratch is refused.  This file
sorts last so a run that stops at the first failure has run everything else.
"""

import ctypes

import pytest
import torch

from suetes_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the float64 kernel tolerance of the parity tests


def _with_workspace(lib, n, nlines, s, c, periodic):
    out = torch.empty_like(s)
    nbytes = int(lib.sisl_ffsl_lines_workspace_bytes(n, nlines))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=s.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.sisl_ffsl_lines(_lib.SISL_F64, n, nlines, s.data_ptr(), c.data_ptr(), periodic, out.data_ptr(),
                             ws.data_ptr(), nbytes, stream)
    assert rc == 0
    return out


def _no_alloc(lib, n, nlines, s, c, periodic):
    out = torch.empty_like(s)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.sisl_ffsl_lines_noalloc(_lib.SISL_F64, n, nlines, s.data_ptr(), c.data_ptr(), periodic,
                                     out.data_ptr(), stream)
    assert rc == 0, _lib.status_string(rc)
    return out


def test_no_alloc_matches_workspace_entry_on_two_calls():
    lib = _lib.load()
    for call, (n, nlines, periodic) in enumerate(((96, 700, 0), (64, 1500, 1))):
        gen = torch.Generator().manual_seed(2024 + call)
        s = (torch.rand(nlines, n, generator=gen, dtype=torch.float64) + 0.1).cuda()
        c = (torch.rand(nlines, n + 1, generator=gen, dtype=torch.float64) - 0.5) * 3.0
        if periodic:  # the two end faces of a periodic line are one face
            c[:, -1] = c[:, 0]
        c = c.cuda()
        got = _no_alloc(lib, n, nlines, s, c, periodic)
        ref = _with_workspace(lib, n, nlines, s, c, periodic)
        torch.cuda.synchronize()
        assert torch.allclose(got, ref, rtol=TOL, atol=TOL), (call, float((got - ref).abs().max()))
        if periodic:  # periodic transport conserves each line's mass
            assert torch.allclose(got.sum(dim=1), s.sum(dim=1), rtol=1e-12)


def test_no_alloc_refuses_more_than_its_scratch():
    lib = _lib.load()
    n = 1023
    nlines = _lib.FFSL_NOALLOC_MAX_DOUBLES // (n + 1) + 1
    s = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.sisl_ffsl_lines_noalloc(_lib.SISL_F64, n, nlines, s.data_ptr(), s.data_ptr(), 0, s.data_ptr(),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.SISL_ERR_SCRATCH_LIMIT
