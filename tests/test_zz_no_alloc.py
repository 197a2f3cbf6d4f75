"""The allocation-free MERBIT entry point, called through the C-ABI.

Some callers cannot call cudaMalloc while they run SpMV (their device memory
belongs to another runtime's pool, or an allocation would synchronise the
device inside a latency-critical loop). mr_spmv_merbit_noalloc keeps its
plan and scratch in a file-scope device array instead. These tests check
that two calls in a row, on different matrices and in FP32, FP16 and BF16
values, give bitwise the y of the planned entry point mr_spmv_merbit and
stay within the SpMV tolerance of the other tests against the FP64 oracle;
that a call leaves the device's free memory unchanged; that a malformed
matrix is refused before any gather; and that sizes beyond the array's
limit are refused. The file is named so that pytest collects it last.
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
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
def test_noalloc_matches_planned_entry_point_on_two_calls(M, O, dtype):
    import torch
    tdt = getattr(torch, dtype)
    f = _noalloc(M)
    stream = torch.cuda.current_stream().cuda_stream
    mats = [M.gen_rmat(scale=14, edge_factor=16, seed=21), M.gen_laplace2d(200, shuffle=True, seed=4)]
    for call, (rp, ci, v) in enumerate(mats):
        vals = _dev(v).to(tdt)
        A = M.view(_dev(rp), _dev(ci), vals)
        xh = M.uniform(rp.size - 1, seed=50 + call)
        x = _dev(xh)
        y_na = torch.full_like(x, float("nan"))
        assert f(C.byref(A), x.data_ptr(), y_na.data_ptr(), stream) == M.MR_OK
        plan = M.MerbitPlan(A)
        y_ref = torch.full_like(x, float("nan"))
        plan.spmv(x, y_ref)
        torch.cuda.synchronize()
        plan.close()
        assert not torch.isnan(y_na).any()
        assert torch.equal(y_na.view(torch.int32), y_ref.view(torch.int32)), (dtype, call)
        # the stored values, widened exactly to FP32, against the FP64 oracle
        stored = vals.float().cpu().numpy()
        ref = O.spmv_f64(rp, ci, stored, xh)
        assert _rel_l2(y_na.cpu().numpy(), ref) <= REL_L2, (dtype, call)


def test_noalloc_call_allocates_no_device_memory(M):
    import torch
    f = _noalloc(M)
    stream = torch.cuda.current_stream().cuda_stream
    # a first call on a small matrix: loads the library's kernels and looks
    # up the static array on this device
    rp, ci, v = M.gen_rmat(scale=10, edge_factor=8, seed=3)
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    x = _dev(M.uniform(rp.size - 1, seed=1))
    y = torch.empty_like(x)
    assert f(C.byref(A), x.data_ptr(), y.data_ptr(), stream) == M.MR_OK
    torch.cuda.synchronize()
    # a larger matrix, all of its buffers made before the measurement
    rp, ci, v = M.gen_rmat(scale=15, edge_factor=16, seed=4)
    B = M.view(_dev(rp), _dev(ci), _dev(v))
    x = _dev(M.uniform(rp.size - 1, seed=2))
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    assert M.lib().mr_release_scratch() == M.MR_OK
    free0, _ = torch.cuda.mem_get_info()
    assert f(C.byref(B), x.data_ptr(), y.data_ptr(), stream) == M.MR_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.isfinite(y).all()


def test_noalloc_rejects_a_malformed_matrix(M):
    import torch
    f = _noalloc(M)
    stream = torch.cuda.current_stream().cuda_stream
    rp, ci, v = M.gen_rmat(scale=10, edge_factor=8, seed=5)
    x = _dev(M.uniform(rp.size - 1, seed=3))
    y = torch.zeros_like(x)
    bad_ci = ci.copy()
    bad_ci[ci.size // 2] = rp.size + 1000  # a column past n_cols
    A = M.view(_dev(rp), _dev(bad_ci), _dev(v))
    assert f(C.byref(A), x.data_ptr(), y.data_ptr(), stream) == M.MR_ERR_INVALID_ARG
    bad_rp = rp.copy()
    bad_rp[5] = bad_rp[6] + 3  # rowptr decreases
    A = M.view(_dev(bad_rp), _dev(ci), _dev(v))
    assert f(C.byref(A), x.data_ptr(), y.data_ptr(), stream) == M.MR_ERR_INVALID_ARG
    torch.cuda.synchronize()
    assert not y.any()  # nothing was written


def test_noalloc_rejects_sizes_beyond_its_scratch(M):
    f = _noalloc(M)
    # n_rows + nnz > 2^24: refused before any device work, pointers unused
    big = M.CsrView(1 << 20, 1 << 20, (1 << 24), 1, 1, 1, M.MR_F32)
    assert f(C.byref(big), 1, 1, None) == M.MR_ERR_UNSUPPORTED
