"""The allocation-free line transport (sisl_ffsl_lines_noalloc).

Callers that cannot call cudaMalloc while they run -- a stream being
captured into a CUDA graph in global mode, a host model that only lends the
library buffers it pre-sized from its own pool, an FFI handler registered
without a workspace -- use this entry point: its float64 scratch is a fixed
8 MiB device array instead of a caller workspace.  The test calls it through
the C ABI twice in a row, with different inputs, in float64 and in float32,
and checks each result against the workspace-taking sisl_ffsl_lines on the
same inputs and against the CPU oracle's FluxFormAdvector.advect_1d
(steppers.py:552-594); it also checks that a problem larger than the fixed
scratch is refused.  This file
sorts last so a run that stops at the first failure has run everything else.
"""

import ctypes

import pytest
import torch

from oracle.steppers import FluxFormAdvector as OracleFFSL
from suetes_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the float64 kernel tolerance of the parity tests
TOL_F32 = 1e-5  # float32 against float64: relative to the line's largest value


def _dtype_code(t):
    return _lib.SISL_F64 if t.dtype == torch.float64 else _lib.SISL_F32


def _with_workspace(lib, n, nlines, s, c, periodic):
    out = torch.empty_like(s)
    nbytes = int(lib.sisl_ffsl_lines_workspace_bytes(n, nlines))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=s.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.sisl_ffsl_lines(_dtype_code(s), n, nlines, s.data_ptr(), c.data_ptr(), periodic, out.data_ptr(),
                             ws.data_ptr(), nbytes, stream)
    assert rc == 0
    return out


def _no_alloc(lib, n, nlines, s, c, periodic):
    out = torch.empty_like(s)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.sisl_ffsl_lines_noalloc(_dtype_code(s), n, nlines, s.data_ptr(), c.data_ptr(), periodic,
                                     out.data_ptr(), stream)
    assert rc == 0, _lib.status_string(rc)
    return out


def _inputs(seed, n, nlines, periodic):
    gen = torch.Generator().manual_seed(seed)
    s = torch.rand(nlines, n, generator=gen, dtype=torch.float64) + 0.1
    c = (torch.rand(nlines, n + 1, generator=gen, dtype=torch.float64) - 0.5) * 3.0
    if periodic:  # the two end faces of a periodic line are one face
        c[:, -1] = c[:, 0]
    return s, c


def test_no_alloc_matches_workspace_entry_on_two_calls():
    lib = _lib.load()
    for call, (n, nlines, periodic) in enumerate(((96, 700, 0), (64, 1500, 1))):
        s, c = _inputs(2024 + call, n, nlines, periodic)
        oracle = OracleFFSL(None, 1.0)._advect_last(s, c, bool(periodic))
        s, c = s.cuda(), c.cuda()
        got = _no_alloc(lib, n, nlines, s, c, periodic)
        ref = _with_workspace(lib, n, nlines, s, c, periodic)
        torch.cuda.synchronize()
        assert torch.allclose(got, ref, rtol=TOL, atol=TOL), (call, float((got - ref).abs().max()))
        err = float((got.cpu() - oracle).abs().max() / oracle.abs().max())
        assert err < TOL, (call, err)
        if periodic:  # periodic transport conserves each line's mass
            assert torch.allclose(got.sum(dim=1), s.sum(dim=1), rtol=1e-12)


def test_no_alloc_float32_matches_workspace_entry_on_two_calls():
    lib = _lib.load()
    for call, (n, nlines, periodic) in enumerate(((80, 900, 0), (48, 2000, 1))):
        s64, c64 = _inputs(77 + call, n, nlines, periodic)
        oracle = OracleFFSL(None, 1.0)._advect_last(s64, c64, bool(periodic))
        s, c = s64.float().cuda(), c64.float().cuda()
        got = _no_alloc(lib, n, nlines, s, c, periodic)
        ref = _with_workspace(lib, n, nlines, s, c, periodic)
        torch.cuda.synchronize()
        # same kernel, same float64 scratch: the two entries agree bitwise
        assert torch.equal(got, ref), (call, float((got - ref).abs().max()))
        err = float((got.double().cpu() - oracle).abs().max() / oracle.abs().max())
        assert err < TOL_F32, (call, err)


def test_no_alloc_refuses_more_than_its_scratch():
    lib = _lib.load()
    n = 1023
    nlines = _lib.FFSL_NOALLOC_MAX_DOUBLES // (n + 1) + 1
    s = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.sisl_ffsl_lines_noalloc(_lib.SISL_F64, n, nlines, s.data_ptr(), s.data_ptr(), 0, s.data_ptr(),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.SISL_ERR_SCRATCH_LIMIT
