"""cfd_residual_norm_noalloc: the residual entry point for callers that cannot
allocate device memory (a solver inside a host application that has already
reserved the device memory, or a latency-critical loop where cudaMalloc would
synchronize the device). It keeps its reduction scratch in a fixed array built
into the library, so this test checks, through the C ABI, that two calls in a
row agree with the allocating path (b minus cfd_spmv's A x, and its norm) and
that inputs beyond the fixed scratch limit are refused.

Collected last on purpose (file name), so a run that stops at the first failure
has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ROWS = 33_546_240  # one partial per 256 rows in 1 MiB of scratch


def _call(torch, A, x, b):
    from cfdrs_b200 import _lib
    rp = torch.as_tensor(A.row_ptr.astype(np.int32), device="cuda")
    col = torch.as_tensor(A.col, device="cuda")
    val = torch.as_tensor(A.val, device="cuda")
    r = torch.empty(A.nrows, dtype=torch.float64, device="cuda")
    n2 = torch.empty(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = _lib.load().cfd_residual_norm_noalloc(
        A.nrows, A.ncols, C.c_void_p(rp.data_ptr()), C.c_void_p(col.data_ptr()), C.c_void_p(val.data_ptr()),
        C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(r.data_ptr()), C.c_void_p(n2.data_ptr()),
        C.c_void_p(stream or 0x1))
    _lib.check(st)
    torch.cuda.synchronize()
    return r, float(n2.item())


def _reference(torch, A, x, b):
    """The allocating path: y = A x through cfd_spmv on a cfd_csr handle."""
    from cfdrs_b200.device import DeviceCsr
    d = DeviceCsr(A)
    y = torch.empty(A.nrows, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    d.spmv(x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    r = b - y
    return r, float((r * r).sum().item())


@pytest.mark.parametrize("case", ["poisson2d", "variable3d"])
def test_noalloc_residual_matches_spmv_twice(cuda, case):
    torch = cuda
    from cfdrs_b200 import problems as P
    if case == "poisson2d":
        A, b = P.poisson_2d_dirichlet(128, seed=0)
    else:
        A, b, _ = P.poisson_3d_variable(40, 4.0, 1.0, seed=3)
    rng = np.random.default_rng(11)
    bd = torch.as_tensor(b, device="cuda")
    for call in range(2):  # the second call reuses the scratch the first one left behind
        x = torch.as_tensor(rng.uniform(-1, 1, A.ncols), device="cuda")
        r, n2 = _call(torch, A, x, bd)
        r_ref, n2_ref = _reference(torch, A, x, bd)
        scale = float(r_ref.abs().max().item())
        np.testing.assert_allclose(r.cpu().numpy(), r_ref.cpu().numpy(), rtol=1e-13, atol=1e-13 * scale,
                                   err_msg=f"call {call}")
        assert abs(n2 - n2_ref) <= 1e-12 * n2_ref, (call, n2, n2_ref)


def test_noalloc_rejects_sizes_beyond_scratch(cuda):
    from cfdrs_b200 import _lib
    L = _lib.load()
    dummy = cuda.zeros(4, dtype=cuda.float64, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    st = L.cfd_residual_norm_noalloc(MAX_ROWS + 1, 10, p, p, p, p, p, p, p, None)
    assert st == 1  # CFD_ERR_DIM
    assert b"scratch limit" in L.cfd_last_error()
