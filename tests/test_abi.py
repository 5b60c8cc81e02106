"""The C ABI library loads here (no GPU needed), exports every function
declared in include/sisl_b200.h, and the ctypes structs match the C layout."""

import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sisl_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sisl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from suetes_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_lib.PROTOTYPES), set(names) ^ set(_lib.PROTOTYPES)


def test_status_strings_and_version():
    from suetes_b200 import _lib
    lib = _lib.load()
    assert lib.sisl_version() >= 1
    assert _lib.status_string(0) == "ok"
    assert "argument" in _lib.status_string(-1)


def test_struct_layout_matches_header(tmp_path):
    import ctypes
    from suetes_b200 import _lib
    src = tmp_path / "sz.c"
    src.write_text('#include "sisl_b200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(SislGrid), sizeof(SislParams),'
                   ' sizeof(SislBackground), sizeof(SislSolveInfo), sizeof(SislState), sizeof(SislRelaxation),'
                   ' sizeof(SislStepInfo), offsetof(SislParams, solver_maxiter)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    got = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    want = [ctypes.sizeof(c) for c in (_lib.SislGrid, _lib.SislParams, _lib.SislBackground, _lib.SislSolveInfo,
                                       _lib.SislState, _lib.SislRelaxation, _lib.SislStepInfo)]
    want.append(_lib.SislParams.solver_maxiter.offset)
    assert got == want


def test_argument_validation_without_gpu():
    """Invalid descriptors are rejected before any CUDA call."""
    import ctypes
    from suetes_b200 import _lib
    lib = _lib.load()
    g = _lib.SislGrid(1, 4, 4, 0, 0, _lib.SISL_F32, 1.0, 1.0, 1.0)  # nx < 2
    p = _lib.SislParams()
    p.solver_restart = 10
    b = _lib.SislBackground()
    h = ctypes.c_void_p()
    assert lib.sisl_core_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(b), None, ctypes.byref(h)) == -1
    assert lib.sisl_step(None, None, None, None, None, 0, None, None) == -1
    assert lib.sisl_field_elems(ctypes.byref(_lib.SislGrid(4, 5, 6, 0, 0, 0, 1.0, 1.0, 1.0)), 1) == 5 * 5 * 6
    # the reverse-mode entry points reject missing arguments the same way
    nul6, nul10 = (ctypes.c_void_p * 6)(), (ctypes.c_void_p * 10)()
    assert lib.sisl_step_vjp(None, None, nul10, None, None, None, None, 0, None, None) == -1
    assert lib.sisl_explicit_tendencies_vjp(None, nul6, nul6, None, nul6, None, 0, None) == -1
    assert lib.sisl_ffsl_advect_vjp(None, None, None, None, None, None, None, None, None, None, None, 0,
                                    None) == -1
    assert lib.sisl_ffsl_lines_vjp(_lib.SISL_F32, 0, 4, None, None, 0, None, None, None, None, 0, None) == -1
    assert lib.sisl_ffsl_lines_vjp_workspace_bytes(16, 8) >= 2 * 17 * 8 * 8
    # a workspace that is absent, short or not 16-byte aligned is refused before
    # any launch (the pointers are never dereferenced on these paths)
    need = lib.sisl_ffsl_lines_workspace_bytes(16, 8)
    fake = ctypes.c_void_p(0x100000)
    for ws, nb in ((None, need), (ctypes.c_void_p(0x200000), need - 8), (ctypes.c_void_p(0x200008), need + 64)):
        assert lib.sisl_ffsl_lines(_lib.SISL_F32, 16, 8, fake, fake, 0, fake, ws, nb, None) == -3
    assert lib.sisl_ffsl_lines_vjp_workspace_bytes(0, 8) == 0
    out = ctypes.c_void_p()
    assert lib.sisl_step_graph_create_taped(0, None, None, None, None, None, None, None, None,
                                            ctypes.byref(out)) == -1
    assert lib.sisl_step_vjp_graph_create(0, None, None, None, None, None, None, None, None, None,
                                          ctypes.byref(out)) == -1


def test_split_and_physics_entries_reject_missing_arguments():
    """The physics-suite step and the split-explicit entries validate their
    arguments before any CUDA call."""
    import ctypes
    from suetes_b200 import _lib
    lib = _lib.load()
    nul4 = (ctypes.c_void_p * 4)()
    st = _lib.SislState()
    assert lib.sisl_step_physics(None, None, None, None, nul4, None, None, 0, None, None) == -1
    assert lib.sisl_step_physics(None, ctypes.byref(st), ctypes.byref(st), None, nul4, None, None, 0, None,
                                 None) == -1
    assert lib.sisl_split_step(None, ctypes.byref(st), ctypes.byref(st), 4, 0.55, 1e-12, None, nul4, None, 0,
                               None) == -1
    assert lib.sisl_split_diagnose(None, None, None, None, None, None, None) == -1
    assert lib.sisl_workspace_bytes(None, _lib.WS_SPLIT) == 0


def test_split_stepper_stage_counts_follow_python_rounding():
    """round(ns/3), round(ns/2), ns acoustic steps (steppers.py:1106-1112):
    Python's round, ties to even, as the C entry's nearbyint."""
    from suetes_b200.split_explicit import SplitExplicitStepper3D

    class Ph:  # the constructor reads only the grid and periodic axes
        class op:
            periodic_axes = ()
        grid = None
    for ns, want in ((1, (1, 1, 1)), (2, (1, 1, 2)), (3, (1, 2, 3)), (5, (2, 2, 5)), (7, (2, 4, 7)),
                     (12, (4, 6, 12))):
        s = SplitExplicitStepper3D(Ph, 1.0, ns)
        assert (s.ns_stage1, s.ns_stage2, s.ns_stage3) == want, ns
        assert abs(s.dtau_stage1 * s.ns_stage1 - 1.0 / 3.0) < 1e-15
