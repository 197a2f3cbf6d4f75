"""Parity of the whole path at the benchmark configurations themselves.

Each test runs the reference's flow (src/main.cu:109-140: gorder4 with
window 5, relabel, then SpMV, checked against SpMV of the original matrix,
src/class.cu:1435-1445) end to end on the GPU through the C-ABI:

  pGOrder (w = 5, vsize from get_width) -> mr_permute_csr (B = P A P^T) ->
  MERBIT (persistent form with the hub cache, and the two-kernel grid form
  at the reference's SIGMA 14 / 256 threads) and plain CSR on B, x' = P x ->
  y = P^T y' -> compared with the FP64 SpMV of the ORIGINAL matrix.

Checked at:
  * R-MAT scale 16, edge factor 16, seed 1 (the small configuration): the
    permutation against the reference's own order_on_cpu, the permuted CSR
    bit for bit against the oracle and against the reference's gather +
    Thrust sort, MERBIT against the reference's merbit_kernel, the exact RD
    histogram of the reordered x stream against the oracle's Fenwick count;
  * the 2048 x 2048 5-point Laplacian with shuffled rows (4.19M rows, 21M
    nonzeros);
  * R-MAT scale 22, edge factor 16, seed 1 (the headline matrix): the
    permuted CSR bit for bit against the oracle and the reference's relabel,
    and every SpMV form against FP64 after the inverse permutation.
FP32 tolerance: relative L2 <= 1e-5, as everywhere in these tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_L2_F32 = 1e-5


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rel_l2(got, ref):
    ref = np.asarray(ref, np.float64)
    return float(np.linalg.norm(np.asarray(got, np.float64) - ref) / np.linalg.norm(ref))


def _flow(M, O, rp, ci, v, x, check_ref_relabel=True):
    """pGOrder -> GPU permutation -> every SpMV form -> inverse permutation;
    returns the permutation, the device CSR of B and the un-permuted results."""
    import torch
    n = rp.size - 1
    n2o = M.pgorder(rp, ci, vsize=0, width=5)
    perm = np.empty(n, np.int32)
    perm[n2o] = np.arange(n, dtype=np.int32)
    pd = _dev(perm)
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    brp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    bci = torch.empty(ci.size, dtype=torch.int32, device="cuda")
    bv = torch.empty(ci.size, dtype=torch.float32, device="cuda")
    M.permute_csr(A, pd, brp, bci, bv)
    torch.cuda.synchronize()
    # B = P A P^T bit for bit against the oracle's restatement
    orp, oci, ov = O.permute_csr(rp, ci, v, perm)
    assert np.array_equal(brp.cpu().numpy(), orp)
    assert np.array_equal(bci.cpu().numpy(), oci)
    assert np.array_equal(bv.cpu().numpy().view(np.uint32), ov.view(np.uint32))
    del orp, oci, ov
    R = O.ref()
    if check_ref_relabel and R is not None:
        # the reference's relabel (gather + GRAPH::sort(false)) on its COO
        # layout: row_ind = our column, col_ind = our row
        rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
        row_ind, col_ind, vals = _dev(ci.copy()), _dev(rows), _dev(v.copy())
        assert R.ref_relabel_sort(n, int(ci.size), row_ind.data_ptr(), col_ind.data_ptr(), vals.data_ptr(),
                                  pd.data_ptr()) == 0
        g_rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(brp.cpu().numpy()))
        assert np.array_equal(col_ind.cpu().numpy(), g_rows)
        assert np.array_equal(row_ind.cpu().numpy(), bci.cpu().numpy())
        assert np.array_equal(vals.cpu().numpy().view(np.uint32), bv.cpu().numpy().view(np.uint32))
        del row_ind, col_ind, vals
    B = M.view(brp, bci, bv)
    xd = _dev(x)
    xp = torch.empty_like(xd)
    M.permute_vector(pd, xd, xp, inverse=False)
    out = {}

    def unpermute(yp):
        y = torch.empty_like(xd)
        M.permute_vector(pd, yp, y, inverse=True)
        torch.cuda.synchronize()
        return y.cpu().numpy()

    for name, kw in (("merbit_persistent_hub", dict(sigma=14, block=1024)),
                     ("merbit_persistent_sigma20", dict(sigma=20, block=1024)),
                     ("merbit_grid_sigma14_256", dict(sigma=14, block=256, hub_cache=False))):
        plan = M.MerbitPlan(B, **kw)
        yp = torch.full_like(xd, float("nan"))
        plan.spmv(xp, yp)
        out[name] = unpermute(yp)
        plan.close()
    yp = torch.full_like(xd, float("nan"))
    M.spmv_csr(B, xp, yp)
    out["csr"] = unpermute(yp)
    return perm, (brp, bci, bv, xp), out


def _check_against_fp64(O, rp, ci, v, x, out):
    ref = O.spmv_f64(rp, ci, v, x)
    for name, y in out.items():
        assert not np.isnan(y).any(), name
        err = _rel_l2(y, ref)
        assert err <= REL_L2_F32, (name, err)


def test_rmat_s16_small_config_end_to_end(M, O):
    import torch
    rp, ci, v = M.gen_rmat(scale=16, edge_factor=16, seed=1)
    n = rp.size - 1
    assert n == 65536
    x = M.uniform(n, seed=1001)
    vs = M.pgorder_width(n, ci.size)
    assert vs == 1024
    R = O.ref()
    if R is not None:
        # the permutation of the reference's own gorder4 host ordering
        n2o = M.pgorder(rp, ci, vsize=0, width=5)
        assert np.array_equal(n2o.view(np.uint32), O.ref_pgorder(rp, ci, vs, 5))
    perm, (brp, bci, bv, xp), out = _flow(M, O, rp, ci, v, x)
    _check_against_fp64(O, rp, ci, v, x, out)
    # the reference's merbit_kernel on the reordered matrix with our plan's
    # descriptors (the same descriptors as its Tile_Kernel, tested elsewhere)
    if R is not None:
        B = M.view(brp, bci, bv)
        plan = M.MerbitPlan(B, sigma=14, block=256, hub_cache=False)
        inf = plan.info()
        yr, zr = torch.zeros(n, device="cuda"), torch.zeros(n, device="cuda")
        ms = ctypes.c_float(0)
        assert R.ref_merbit_spmv(brp.data_ptr(), bci.data_ptr(), bv.data_ptr(), n, int(ci.size), inf.tile_x_dev,
                                 inf.tile_y_dev, inf.lane_desc_dev, xp.data_ptr(), yr.data_ptr(), zr.data_ptr(), 1,
                                 ctypes.byref(ms)) == 0
        ours = torch.empty_like(yr)
        plan.spmv(xp, ours)
        torch.cuda.synchronize()
        plan.close()
        assert _rel_l2(ours.cpu().numpy(), yr.cpu().numpy()) <= 2 * REL_L2_F32
    # exact reuse-distance histogram of the reordered x stream (log2 bins)
    edges = [1 << k for k in range(21)]
    counts, valid = M.rd_hist_exact(bci, n, sector=32, edges=edges)
    o_counts, o_valid = O.rd_hist_exact(bci.cpu().numpy(), n, 32, edges)
    assert valid == o_valid and np.array_equal(np.asarray(counts), o_counts)


def test_laplace2d_2048_shuffled_config_end_to_end(M, O):
    rp, ci, v = M.gen_laplace2d(2048, shuffle=True, seed=1)
    n = rp.size - 1
    assert n == 2048 * 2048
    x = M.uniform(n, seed=1001)
    _, _, out = _flow(M, O, rp, ci, v, x)
    _check_against_fp64(O, rp, ci, v, x, out)


def test_rmat_s22_headline_config_end_to_end(M, O):
    rp, ci, v = M.gen_rmat(scale=22, edge_factor=16, seed=1)
    n = rp.size - 1
    assert n == 1 << 22
    x = M.uniform(n, seed=1001)
    _, _, out = _flow(M, O, rp, ci, v, x)
    _check_against_fp64(O, rp, ci, v, x, out)
