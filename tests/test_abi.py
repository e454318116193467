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


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _i64(*v):
    import numpy as np
    return np.array(v, dtype=np.int64)


def test_csr_row_ptr_past_nnz_is_refused_before_the_column_scan():
    """row_ptr = [0, 100, 5] with 5 nonzeros: row 0's end passes nnz. The
    check must fire at row 0, before the column scan reads col[5..99]
    (without it the call still fails, but on a column it read past the end)."""
    import numpy as np
    from cfdrs_b200 import _lib
    L = _lib.load()
    rp, col, val = _i64(0, 100, 5), np.arange(5, dtype=np.int32), np.ones(5)
    x, y = np.ones(8), np.zeros(2)
    info = (C.c_int64 * 64)()
    st = L.cfd_layout_check(2, 8, 5, _ptr(rp), _ptr(col), _ptr(val), _ptr(x), _ptr(y), C.byref(info))
    assert st == 1 and b"passes nnz at row 0" in L.cfd_last_error()
    cfg = _lib.AmgConfigC()
    L.cfd_amg_config_default(C.byref(cfg))
    out = C.c_void_p()
    col64 = np.arange(5, dtype=np.int64)
    assert L.cfd_amg_setup_host(2, _ptr(rp), _ptr(col64), _ptr(val), C.byref(cfg), C.byref(out)) == 1
    assert b"passes nnz at row 0" in L.cfd_last_error() and not out.value


BATCH_LAYOUTS = {
    # name: (num_systems, offsets, row_ptr, col, with_values, status, message)
    "null_offsets": (0, None, _i64(0), None, False, 7, b"invalid arguments"),
    "negative_count": (-1, _i64(0), _i64(0), None, False, 7, b"invalid arguments"),
    "negative_rows": (1, _i64(0, -5), _i64(0), None, False, 1, b"system offsets must start at 0"),
    "offsets_not_from_zero": (1, _i64(1, 2), _i64(0, 1, 2), None, False, 1, b"system offsets must start at 0"),
    # system 0 claims 100 rows of a 50-row batch: row_ptr[100] must not be read
    "offsets_decrease": (2, _i64(0, 100, 50), _i64(*range(51)), "diag", True, 1, b"decrease or pass the row count"),
    "row_ptr_past_nnz": (1, _i64(0, 2), _i64(0, 100, 2), "diag", True, 1, b"passes nnz at row 0"),
    "null_columns": (1, _i64(0, 2), _i64(0, 1, 2), None, True, 1, b"null column or value array"),
    "null_values": (1, _i64(0, 2), _i64(0, 1, 2), "diag", False, 1, b"null column or value array"),
    "local_column_out_of_range": (2, _i64(0, 2, 4), _i64(0, 1, 2, 3, 4), "global", True, 1, b"local column 2"),
    "system_too_large": (1, _i64(0, 2049), _i64(*range(2050)), "diag", True, 1, b"at most 2048 rows"),
}


@pytest.mark.parametrize("case", sorted(BATCH_LAYOUTS))
def test_batch_layout_is_checked_before_the_context(case):
    """cfd_batch_create checks the caller's layout before it touches the
    context, in an order that reads no array past a bound an earlier check
    established; a null context is reported only for a valid layout."""
    import numpy as np
    from cfdrs_b200 import _lib
    L = _lib.load()
    nsys, offs, rp, col, with_values, status, msg = BATCH_LAYOUTS[case]
    nnz = int(rp[-1]) if rp is not None and rp[-1] >= 0 else 0
    cols = None
    if col == "diag":          # local column = the row's index inside its system
        cols = np.array([i - offs[np.searchsorted(offs, i, side="right") - 1] for i in range(nnz)], dtype=np.int32)
    elif col == "global":      # global row numbers: system 1's columns leave its 2 rows
        cols = np.arange(nnz, dtype=np.int32)
    vals = np.ones(nnz) if with_values else None
    out = C.c_void_p(1)
    st = L.cfd_batch_create(None, nsys, _ptr(offs), _ptr(rp), _ptr(cols), _ptr(vals), C.byref(out))
    assert st == status, L.cfd_last_error()
    assert msg in L.cfd_last_error() and not out.value


def test_batch_valid_layout_reaches_the_context_check():
    import numpy as np
    from cfdrs_b200 import _lib
    L = _lib.load()
    out = C.c_void_p()
    offs, rp = _i64(0, 2, 2, 5), _i64(0, 1, 2, 3, 4, 5)   # system 1 is empty
    cols, vals = np.array([0, 1, 0, 1, 2], dtype=np.int32), np.ones(5)
    assert L.cfd_batch_create(None, 3, _ptr(offs), _ptr(rp), _ptr(cols), _ptr(vals), C.byref(out)) == 7
    assert b"null context" in L.cfd_last_error()
    z = _i64(0)
    assert L.cfd_batch_create(None, 0, _ptr(z), _ptr(z), None, None, C.byref(out)) == 7
    assert b"null context" in L.cfd_last_error()


HOST_OOM_SCRIPT = r"""
import ctypes as C, resource, sys
import numpy as np
from cfdrs_b200 import _lib
from cfdrs_b200 import problems as P
L = _lib.load()
A = P.poisson_3d_variable(40, 4.0, 1.0, seed=1)[0]
rp, col = np.ascontiguousarray(A.row_ptr, np.int64), np.ascontiguousarray(A.col, np.int64)
val = np.ascontiguousarray(A.val)
cfg = _lib.AmgConfigC()
L.cfd_amg_config_default(C.byref(cfg))
vm = int([l for l in open("/proc/self/status") if l.startswith("VmSize")][0].split()[1]) * 1024
resource.setrlimit(resource.RLIMIT_AS, (vm + (8 << 20), resource.RLIM_INFINITY))
out = C.c_void_p()
st = L.cfd_amg_setup_host(A.nrows, rp.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                          val.ctypes.data_as(C.c_void_p), C.byref(cfg), C.byref(out))
resource.setrlimit(resource.RLIMIT_AS, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
print(st, L.cfd_last_error().decode(), out.value is None)
"""


@pytest.mark.skipif(not os.path.exists("/proc/self/status"), reason="needs /proc for the address-space size")
@pytest.mark.skipif("libasan" in os.environ.get("LD_PRELOAD", ""),
                    reason="the sanitizer's allocator aborts on exhaustion instead of throwing std::bad_alloc")
def test_host_allocation_failure_is_a_status():
    """A host allocation that fails inside an entry point comes back as
    CFD_ERR_ALLOC with no handle, and the caller's process carries on (an
    exception unwinding out of the C ABI would end it with std::terminate).
    The child caps its address space at 8 MiB above its size before the host
    AMG setup of a 40^3 operator; one OpenMP thread, so that no thread is
    created under the cap."""
    import sys
    env = dict(os.environ, OMP_NUM_THREADS="1", PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", HOST_OOM_SCRIPT], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    st, rest = out.stdout.strip().split(" ", 1)
    assert int(st) == 6 and "host memory allocation failed" in rest and rest.endswith("True")
