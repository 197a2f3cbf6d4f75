"""The allocation-free MERBIT entry point, called through the C-ABI.

Some callers cannot call cudaMalloc while they run SpMV (their device memory
belongs to another runtime's pool, or an allocation would synchronise the
device inside a latency-critical loop). mr_spmv_merbit_noalloc keeps its
plan and scratch in a file-scope device array instead. This test checks that
two calls in a row, on different matrices, give the same y as the planned
entry point mr_spmv_merbit within the SpMV tolerance of the other tests, and
that sizes beyond the array's limit are refused. It lives in its own file so
that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_L2 = 1e-5


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _noalloc(M):
    L = M.lib()
    f = L.mr_spmv_merbit_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(M.CsrView), C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def _rel_l2(a, b):
    a = a.double()
    b = b.double()
    return float((a - b).norm() / b.norm())


def test_noalloc_matches_planned_entry_point_on_two_calls(M):
    import torch
    f = _noalloc(M)
    stream = torch.cuda.current_stream().cuda_stream
    mats = [M.gen_rmat(scale=14, edge_factor=16, seed=21), M.gen_laplace2d(200, shuffle=True, seed=4)]
    for call, (rp, ci, v) in enumerate(mats):
        A = M.view(_dev(rp), _dev(ci), _dev(v))
        x = _dev(M.uniform(rp.size - 1, seed=50 + call))
        y_na = torch.full_like(x, float("nan"))
        assert f(C.byref(A), x.data_ptr(), y_na.data_ptr(), stream) == M.MR_OK
        plan = M.MerbitPlan(A)
        y_ref = torch.full_like(x, float("nan"))
        plan.spmv(x, y_ref)
        torch.cuda.synchronize()
        assert not torch.isnan(y_na).any()
        assert _rel_l2(y_na, y_ref) <= REL_L2, call
        plan.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(M):
    f = _noalloc(M)
    # n_rows + nnz > 2^24: refused before any device work, pointers unused
    big = M.CsrView(1 << 20, 1 << 20, (1 << 24), 1, 1, 1, M.MR_F32)
    assert f(C.byref(big), 1, 1, None) == M.MR_ERR_UNSUPPORTED
