"""GPU parity of the SpMV path: MERBIT plan descriptors (bit-exact against the
oracle's restatement of Tile_Kernel and, when built, the reference kernel
itself), MERBIT and plain CSR SpMV against the FP64 oracle (relative L2
<= 1e-5 for FP32 values), determinism, dtypes and edge cases."""
import numpy as np
import pytest

from conftest import csr_from_dense_pattern, csr_random

pytestmark = pytest.mark.gpu

REL_L2_F32 = 1e-5


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rel_l2(got, ref):
    ref = np.asarray(ref, np.float64)
    d = np.linalg.norm(np.asarray(got, np.float64) - ref)
    nr = np.linalg.norm(ref)
    return d / nr if nr > 0 else d


def _plan_and_spmv(M, rp, ci, v, x, sigma=14, block=0, dtype=None):
    import torch
    vals = _dev(v)
    if dtype is not None:
        vals = vals.to(dtype)
    ncols = max(rp.size - 1, int(ci.max(initial=0)) + 1)
    A = M.view(_dev(rp), _dev(ci), vals, n_cols=ncols)
    keep = (A, vals)
    plan = M.MerbitPlan(A, sigma=sigma, block=block)
    xd = _dev(x)
    y = torch.full((rp.size - 1,), float("nan"), device="cuda")
    plan.spmv(xd, y)
    torch.cuda.synchronize()
    return plan, y.cpu().numpy(), keep


def _edge_cases():
    rng = np.random.default_rng(0)
    cases = {
        "one_row": csr_from_dense_pattern([[0]]),
        "one_row_empty": csr_from_dense_pattern([[]]),
        "all_empty": csr_from_dense_pattern([[] for _ in range(1000)]),
        "single_nnz": csr_from_dense_pattern([[] for _ in range(500)] + [[7]] + [[] for _ in range(499)]),
        "huge_row": csr_from_dense_pattern([sorted(rng.choice(60000, 50000, replace=False).tolist())] +
                                           [[i] for i in range(1, 300)]),
        "rows_fill_lane": csr_from_dense_pattern([[j for j in range(13)] for _ in range(700)]),
        "rows_fill_tile": csr_from_dense_pattern([[j for j in range(447)] for _ in range(40)]),
        "rows_fill_block": csr_from_dense_pattern([[j for j in range(3583)] for _ in range(6)]),
        "random_small": csr_random(3000, 40, seed=1, empty_frac=0.2),
        "random_wide": csr_random(2000, 300, seed=2, ncols=5000, empty_frac=0.5),
        # row lengths around the plain CSR kernel's 2048-nonzero slices and
        # its 4096 long-row cut, long rows back to back, empty rows between
        # them, and trailing empty rows after a nonzero count that is a
        # multiple of the slice
        "slice_edges": csr_from_dense_pattern(
            [list(range(L)) for L in (2048, 0, 0, 4096, 4097, 1, 2047, 2049, 0, 4097, 4097, 12000, 3, 0)]),
        "slice_multiple": csr_from_dense_pattern([list(range(1024)) for _ in range(4)] + [[] for _ in range(100)]),
    }
    return cases


@pytest.fixture(scope="module")
def cases(M):
    c = _edge_cases()
    rp, ci, v = M.gen_rmat(scale=13, edge_factor=16, seed=4)
    c["rmat13"] = (rp, ci, v)
    rp, ci, v = M.gen_laplace2d(64, shuffle=True, seed=3)
    c["lap64"] = (rp, ci, v)
    return c


@pytest.mark.parametrize("sigma", [7, 14, 16, 32])
def test_plan_descriptors_match_oracle(M, O, cases, sigma):
    for name, (rp, ci, v) in cases.items():
        plan, _, _ = _plan_and_spmv(M, rp, ci, v, np.ones(max(rp.size - 1, int(ci.max(initial=0)) + 1), np.float32),
                                    sigma=sigma)
        tx, ty, ld = plan.descriptors()
        otx, oty, old = O.merbit_plan(rp, ci.size, sigma)
        assert np.array_equal(tx, otx), (name, sigma, "tile_x")
        assert np.array_equal(ty, oty), (name, sigma, "tile_y")
        assert np.array_equal(ld, old), (name, sigma, "lane_desc")
        plan.close()


def test_plan_descriptors_match_reference_kernel(M, O, cases):
    R = O.ref()
    if R is None:
        pytest.skip("reference build (oracle/_ref) not present")
    import torch
    for name, (rp, ci, v) in cases.items():
        n = rp.size - 1
        plan, _, _ = _plan_and_spmv(M, rp, ci, v, np.ones(max(n, int(ci.max(initial=0)) + 1), np.float32))
        tx, ty, ld = plan.descriptors()
        rtx = torch.zeros(tx.size, dtype=torch.int32, device="cuda")
        rty = torch.zeros(ty.size, dtype=torch.int32, device="cuda")
        rld = torch.zeros(max(ld.size, 1), dtype=torch.int32, device="cuda")
        rpd = _dev(rp)
        assert R.ref_tile_build(rpd.data_ptr(), n, int(ci.size), rtx.data_ptr(), rty.data_ptr(), rld.data_ptr()) == 0
        assert np.array_equal(tx, rtx.cpu().numpy().view(np.uint32)), name
        assert np.array_equal(ty, rty.cpu().numpy().view(np.uint32)), name
        assert np.array_equal(ld, rld.cpu().numpy().view(np.uint32)[:ld.size]), name
        plan.close()


@pytest.mark.parametrize("sigma", [7, 10, 14, 16, 20, 24, 28, 32])
def test_merbit_spmv_matches_fp64(M, O, cases, sigma):
    for name, (rp, ci, v) in cases.items():
        ncols = max(rp.size - 1, int(ci.max(initial=0)) + 1)
        x = M.uniform(ncols, seed=11)
        plan, y, _ = _plan_and_spmv(M, rp, ci, v, x, sigma=sigma)
        ref = O.spmv_f64(rp, ci, v, x)
        assert not np.isnan(y).any(), (name, sigma)
        assert _rel_l2(y, ref) <= REL_L2_F32, (name, sigma, _rel_l2(y, ref))
        plan.close()


@pytest.mark.parametrize("block", [128, 256, 512, 1024])
def test_merbit_block_sizes(M, O, cases, block):
    """Every form (grid kernels of 4 / 8 / 16 warps with the separate fix-up
    kernel, and the persistent kernel with its fused fix-up) against FP64,
    and bit for bit against the persistent form, on every edge case (huge
    rows give carry runs that span many CTAs); repeated launches of one plan
    give the same bits (the persistent kernel's arrival counters and ticket
    reset themselves)."""
    import torch
    for name, (rp, ci, v) in cases.items():
        ncols = max(rp.size - 1, int(ci.max(initial=0)) + 1)
        x = M.uniform(ncols, seed=5)
        for sigma in (7, 14, 20):
            plan, y, _ = _plan_and_spmv(M, rp, ci, v, x, sigma=sigma, block=block)
            ref_plan, y_ref, _ = _plan_and_spmv(M, rp, ci, v, x, sigma=sigma, block=1024)
            assert _rel_l2(y, O.spmv_f64(rp, ci, v, x)) <= REL_L2_F32, (name, sigma)
            assert np.array_equal(y.view(np.int32), y_ref.view(np.int32)), (name, sigma)
            y2 = torch.full((rp.size - 1,), float("nan"), device="cuda")
            for _ in range(2):
                plan.spmv(_dev(x), y2)
            torch.cuda.synchronize()
            assert np.array_equal(y2.cpu().numpy().view(np.int32), y.view(np.int32)), (name, sigma)
            plan.close()
            ref_plan.close()


@pytest.mark.parametrize("sigma", [7, 14, 32])
def test_persistent_and_two_kernel_forms_bit_identical(M, cases, sigma):
    """The persistent kernel finishes carry runs inside its chunk and at chunk
    boundaries; the two-kernel form in one fix-up pass. Both sum each run in
    FP64 in tile order, so they must agree bit for bit."""
    import torch
    rp, ci, v = M.gen_rmat(scale=17, edge_factor=16, seed=8)
    big = dict(cases)
    big["rmat17"] = (rp, ci, v)
    # 1,050,000 empty rows, then 10 rows of 1,300 nonzeros: the cost-balanced
    # chunks of the persistent kernel are empty around each dense tile (17 to
    # 54 of them, by SIGMA, on 148 SMs), and the dense rows' carry runs cross
    # those empty chunks
    rng = np.random.default_rng(4)
    ne, nd, L = 1050000, 10, 1300
    lens = np.concatenate([np.zeros(ne, np.int64), np.full(nd, L, np.int64)])
    rp_d = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci_d = np.concatenate([np.sort(rng.choice(ne + nd, L, replace=False)) for _ in range(nd)]).astype(np.int32)
    big["empty_then_dense"] = (rp_d, ci_d, rng.uniform(-1, 1, ci_d.size).astype(np.float32))
    for name, (rp, ci, v) in big.items():
        ncols = max(rp.size - 1, int(ci.max(initial=0)) + 1)
        x = M.uniform(ncols, seed=2)
        p1, y1, _ = _plan_and_spmv(M, rp, ci, v, x, sigma=sigma, block=1024)
        p2, y2, _ = _plan_and_spmv(M, rp, ci, v, x, sigma=sigma, block=256)
        assert np.array_equal(y1.view(np.int32), y2.view(np.int32)), (name, sigma)
        p1.close()
        p2.close()


def test_persistent_plan_replays_in_cuda_graph(M):
    """The persistent kernel's completion ticket and chunk-boundary counters
    are reset by the launch that uses them: a captured SpMV replayed many
    times (and mixed with direct calls) gives the direct call's y bit for
    bit every time."""
    import torch
    rp, ci, v = M.gen_rmat(scale=17, edge_factor=16, seed=8)
    n = rp.size - 1
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    x = _dev(M.uniform(n, seed=6))
    plan = M.MerbitPlan(A, sigma=14, block=1024)
    ref = torch.empty_like(x)
    plan.spmv(x, ref)
    torch.cuda.synchronize()
    y = torch.full_like(x, float("nan"))
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        plan.spmv(x, y, stream=s)  # warm-up on the capture stream
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        plan.spmv(x, y, stream=torch.cuda.current_stream())
    for k in range(20):
        y.fill_(float("nan"))
        g.replay()
        if k % 5 == 4:
            plan.spmv(x, y)  # direct calls between replays
        torch.cuda.synchronize()
        assert torch.equal(y.view(torch.int32), ref.view(torch.int32)), k
    del g
    plan.close()


def test_hub_cache_bit_identical_and_reported(M):
    """The shared-memory hub cache changes where x comes from, not the
    arithmetic: results must equal the plan without it bit for bit. Skewed
    R-MAT columns get a cache; a large banded matrix (no hot columns) not."""
    import torch
    rp, ci, v = M.gen_rmat(scale=18, edge_factor=16, seed=12)
    n = rp.size - 1
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    x = _dev(M.uniform(n, seed=3))
    hub = M.MerbitPlan(A)
    plain = M.MerbitPlan(A, hub_cache=False)
    inf = hub.info()
    assert inf.hub_columns > 0 and inf.hub_coverage >= 0.25
    assert plain.info().hub_columns == 0
    y1 = torch.empty_like(x)
    y2 = torch.empty_like(x)
    for _ in range(2):
        hub.spmv(x, y1)
        plain.spmv(x, y2)
    torch.cuda.synchronize()
    assert torch.equal(y1.view(torch.int32), y2.view(torch.int32))
    # the descriptors are the reference format either way
    assert all(np.array_equal(a, b) for a, b in zip(hub.descriptors(), plain.descriptors()))
    hub.close()
    plain.close()
    rp, ci, v = M.gen_banded(1 << 20, 9, seed=1)
    B = M.view(_dev(rp), _dev(ci), _dev(v))
    assert M.MerbitPlan(B).info().hub_columns == 0


def test_merbit_is_deterministic(M, cases):
    import torch
    rp, ci, v = cases["huge_row"]
    ncols = int(ci.max()) + 1
    x = M.uniform(ncols, seed=3)
    vals = _dev(v)
    A = M.view(_dev(rp), _dev(ci), vals, n_cols=ncols)
    plan = M.MerbitPlan(A)
    xd = _dev(x)
    y1 = torch.empty(rp.size - 1, device="cuda")
    y2 = torch.empty(rp.size - 1, device="cuda")
    plan.spmv(xd, y1)
    for _ in range(3):
        plan.spmv(xd, y2)
    torch.cuda.synchronize()
    assert torch.equal(y1.view(torch.int32), y2.view(torch.int32))
    plan.close()


@pytest.mark.parametrize("tdt", ["float16", "bfloat16"])
def test_merbit_half_values(M, O, cases, tdt):
    import torch
    dt = getattr(torch, tdt)
    for name in ("rmat13", "huge_row", "random_small"):
        rp, ci, v = cases[name]
        ncols = max(rp.size - 1, int(ci.max(initial=0)) + 1)
        x = M.uniform(ncols, seed=13)
        plan, y, _ = _plan_and_spmv(M, rp, ci, v, x, dtype=dt)
        v_rounded = torch.from_numpy(v).to(dt).float().numpy()
        assert _rel_l2(y, O.spmv_f64(rp, ci, v_rounded, x)) <= REL_L2_F32, (name, tdt)
        plan.close()


def test_merbit_vs_reference_kernel(M, O, cases):
    R = O.ref()
    if R is None:
        pytest.skip("reference build (oracle/_ref) not present")
    import ctypes
    import torch
    for name in ("rmat13", "lap64", "random_small", "rows_fill_tile"):
        rp, ci, v = cases[name]
        n = rp.size - 1
        x = M.uniform(max(n, int(ci.max(initial=0)) + 1), seed=21)
        plan, y, _ = _plan_and_spmv(M, rp, ci, v, x)
        inf = plan.info()
        yr = torch.zeros(n, device="cuda")
        zr = torch.zeros(n, device="cuda")
        rpd, cid, vd, xd = _dev(rp), _dev(ci), _dev(v), _dev(x)
        ms = ctypes.c_float(0)
        assert R.ref_merbit_spmv(rpd.data_ptr(), cid.data_ptr(), vd.data_ptr(), n, int(ci.size), inf.tile_x_dev,
                                 inf.tile_y_dev, inf.lane_desc_dev, xd.data_ptr(), yr.data_ptr(), zr.data_ptr(), 3,
                                 ctypes.byref(ms)) == 0
        ref64 = O.spmv_f64(rp, ci, v, x)
        assert _rel_l2(yr.cpu().numpy(), ref64) <= REL_L2_F32, name
        assert _rel_l2(y, yr.cpu().numpy()) <= 2 * REL_L2_F32, name
        plan.close()


@pytest.mark.parametrize("tdt", ["float32", "float16", "bfloat16"])
def test_csr_spmv_matches_fp64(M, O, cases, tdt):
    import torch
    dt = getattr(torch, tdt)
    for name, (rp, ci, v) in cases.items():
        ncols = max(rp.size - 1, int(ci.max(initial=0)) + 1)
        x = M.uniform(ncols, seed=17)
        vals = _dev(v).to(dt)
        A = M.view(_dev(rp), _dev(ci), vals, n_cols=ncols)
        y = torch.full((rp.size - 1,), float("nan"), device="cuda")
        M.spmv_csr(A, _dev(x), y)
        torch.cuda.synchronize()
        vr = vals.float().cpu().numpy()
        assert _rel_l2(y.cpu().numpy(), O.spmv_f64(rp, ci, vr, x)) <= REL_L2_F32, (name, tdt)


def test_csr_spmv_is_deterministic(M, cases):
    import torch
    for name in ("huge_row", "slice_edges", "rmat13"):
        rp, ci, v = cases[name]
        ncols = max(rp.size - 1, int(ci.max(initial=0)) + 1)
        A = M.view(_dev(rp), _dev(ci), _dev(v), n_cols=ncols)
        x = _dev(M.uniform(ncols, seed=5))
        ys = []
        for _ in range(3):
            y = torch.empty(rp.size - 1, device="cuda")
            M.spmv_csr(A, x, y)
            ys.append(y)
        torch.cuda.synchronize()
        assert all(torch.equal(ys[0].view(torch.int32), t.view(torch.int32)) for t in ys[1:]), name


def test_plan_rejects_mismatched_matrix(M, cases):
    rp, ci, v = cases["rmat13"]
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    plan = M.MerbitPlan(A)
    rp2, ci2, v2 = cases["lap64"]
    B = M.view(_dev(rp2), _dev(ci2), _dev(v2))
    import torch
    with pytest.raises(M.MRError) as e:
        plan.spmv(_dev(np.ones(rp2.size - 1, np.float32)), torch.empty(rp2.size - 1, device="cuda"), A=B)
    assert e.value.code == M.MR_ERR_INVALID_ARG
    plan.close()
