"""The C-ABI library loads and exports every entry point include/cfdgpu.h declares."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cfdgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cfd_[a-z0-9_]+)\s*\(", src)))


def test_header_matches_binding_table():
    from cfdrs_b200 import _lib
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    from cfdrs_b200 import _lib
    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (cfd_[a-z0-9_]+)", out))
    assert set(declared_functions()) <= exported


def test_defaults_and_version():
    from cfdrs_b200 import _lib
    L = _lib.load()
    assert L.cfd_version().decode().startswith("cfdgpu")
    c = _lib.AmgConfigC()
    L.cfd_amg_config_default(C.byref(c))
    assert (c.max_levels, c.min_coarse_size, c.pre_smooth, c.post_smooth) == (10, 50, 2, 2)
    assert c.strength_threshold == 0.25 and c.relaxation == 1.0 and c.coarse_sweeps == 10
    o = _lib.SolveOptionsC()
    L.cfd_solve_options_default(C.byref(o))
    assert o.inner_tolerance == 1e-4


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from cfdrs_b200 import _lib
    L = _lib.load()
    h = C.c_void_p()
    st = L.cfd_context_create(0, C.byref(h))
    assert st != _lib.CFD_OK and L.cfd_last_error()
    with pytest.raises(_lib.CfdError):
        _lib.check(st)
