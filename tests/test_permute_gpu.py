"""GPU parity of the permutation application: B = P A P^T must equal the
oracle's restatement bit for bit (rowptr, colidx and value bits) and, when
built, the reference's own gather + GRAPH::sort(false) relabel; invalid
permutations are reported; the whole reorder -> MERBIT -> inverse-permute
flow matches the FP64 SpMV of the original matrix."""
import numpy as np
import pytest

from conftest import csr_from_dense_pattern, csr_random

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _permute(M, rp, ci, v, perm, dtype=None):
    import torch
    vals = _dev(v)
    if dtype is not None:
        vals = vals.to(dtype)
    A = M.view(_dev(rp), _dev(ci), vals)
    orp = torch.empty(rp.size, dtype=torch.int32, device="cuda")
    oci = torch.empty(max(ci.size, 1), dtype=torch.int32, device="cuda")
    ov = torch.empty(max(ci.size, 1), dtype=vals.dtype, device="cuda")
    M.permute_csr(A, _dev(perm), orp, oci, ov)
    torch.cuda.synchronize()
    return orp.cpu().numpy(), oci.cpu().numpy()[:ci.size], ov.cpu()[:ci.size]


def _heavy_rows(seed=0):
    rng = np.random.default_rng(seed)
    n = 60000
    rows = [[] for _ in range(n)]
    for r, k in ((5, 20000), (17, 4097), (400, 9000), (59999, 33000), (1000, 4096), (1001, 33), (1002, 32)):
        rows[r] = sorted(rng.choice(n, k, replace=False).tolist())
    for r in range(2000, 2600):
        rows[r] = sorted(rng.choice(n, int(rng.integers(1, 300)), replace=False).tolist())
    return csr_from_dense_pattern(rows)


def _duplicate_columns(seed=1):
    """Rows that repeat column indices, one per sort class (warp, warp x2/4/8
    keys, CTA, long-row merge): equal new columns must keep source order."""
    rng = np.random.default_rng(seed)
    n = 12000
    rows = [[] for _ in range(n)]
    for r, k in ((3, 20), (50, 60), (51, 100), (52, 250), (700, 1000), (701, 4096), (9000, 5000), (9001, 11000)):
        rows[r] = rng.choice(max(k // 3, 2), k, replace=True).tolist()  # unsorted, many repeats
    return csr_from_dense_pattern(rows)


@pytest.fixture(scope="module")
def mats(M):
    return {
        "rmat14": M.gen_rmat(scale=14, edge_factor=16, seed=2),
        "lap48": M.gen_laplace2d(48, shuffle=True, seed=1),
        "heavy": _heavy_rows(),
        "random": csr_random(5000, 70, seed=8, empty_frac=0.3),
        "tiny": csr_from_dense_pattern([[1], [0, 1], []]),
        "dups": _duplicate_columns(),
    }


@pytest.mark.parametrize("name", ["rmat14", "lap48", "heavy", "random", "tiny", "dups"])
def test_permute_bit_exact_vs_oracle(M, O, mats, name):
    rp, ci, v = mats[name]
    n = rp.size - 1
    perm = M.random_perm(n, seed=99)
    grp, gci, gv = _permute(M, rp, ci, v, perm)
    orp, oci, ov = O.permute_csr(rp, ci, v, perm)
    assert np.array_equal(grp, orp)
    assert np.array_equal(gci, oci)
    assert np.array_equal(gv.numpy().view(np.uint32), ov.view(np.uint32))


@pytest.mark.parametrize("tdt", ["float16", "bfloat16"])
def test_permute_half_values(M, O, mats, tdt):
    import torch
    rp, ci, v = mats["heavy"]
    perm = M.random_perm(rp.size - 1, seed=5)
    dt = getattr(torch, tdt)
    grp, gci, gv = _permute(M, rp, ci, v, perm, dtype=dt)
    vr = torch.from_numpy(v).to(dt).float().numpy()
    orp, oci, ov = O.permute_csr(rp, ci, vr, perm)
    assert np.array_equal(grp, orp) and np.array_equal(gci, oci)
    assert np.array_equal(gv.float().numpy(), ov)


def test_permute_identity_and_pgorder(M, O, mats):
    rp, ci, v = mats["rmat14"]
    n = rp.size - 1
    grp, gci, gv = _permute(M, rp, ci, v, np.arange(n, dtype=np.int32))
    assert np.array_equal(grp, rp) and np.array_equal(gci, ci) and np.array_equal(gv.numpy(), v)
    p_n2o = M.pgorder(rp, ci, 0, 5)
    perm = np.empty(n, np.int32)
    perm[p_n2o] = np.arange(n, dtype=np.int32)
    grp, gci, gv = _permute(M, rp, ci, v, perm)
    orp, oci, ov = O.permute_csr(rp, ci, v, perm)
    assert np.array_equal(grp, orp) and np.array_equal(gci, oci) and np.array_equal(gv.numpy(), ov)


def test_permute_vs_reference_relabel(M, O, mats):
    R = O.ref()
    if R is None:
        pytest.skip("reference build (oracle/_ref) not present")
    import torch
    for name in ("rmat14", "heavy", "lap48"):
        rp, ci, v = mats[name]
        n = rp.size - 1
        perm = M.random_perm(n, seed=123)
        rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
        # reference layout: row_ind = our column, col_ind = our row
        row_ind, col_ind, vals = _dev(ci.copy()), _dev(rows), _dev(v.copy())
        assert R.ref_relabel_sort(n, int(ci.size), row_ind.data_ptr(), col_ind.data_ptr(), vals.data_ptr(),
                                  _dev(perm).data_ptr()) == 0
        r_cols = row_ind.cpu().numpy()
        r_rows = col_ind.cpu().numpy()
        r_vals = vals.cpu().numpy()
        grp, gci, gv = _permute(M, rp, ci, v, perm)
        g_rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(grp))
        assert np.array_equal(g_rows, r_rows), name
        assert np.array_equal(gci, r_cols), name
        assert np.array_equal(gv.numpy().view(np.uint32), r_vals.view(np.uint32)), name


def test_invalid_permutations_rejected(M, mats):
    import torch
    rp, ci, v = mats["random"]
    n = rp.size - 1
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    out = (torch.empty(n + 1, dtype=torch.int32, device="cuda"), torch.empty(ci.size, dtype=torch.int32, device="cuda"),
           torch.empty(ci.size, dtype=torch.float32, device="cuda"))
    dup = np.arange(n, dtype=np.int32)
    dup[3] = dup[4]
    oob = np.arange(n, dtype=np.int32)
    oob[7] = n + 5
    neg = np.arange(n, dtype=np.int32)
    neg[0] = -1
    for bad in (dup, oob, neg):
        with pytest.raises(M.MRError) as e:
            M.permute_csr(A, _dev(bad), *out)
        assert e.value.code == M.MR_ERR_INVALID_PERM
        assert not M.check_perm(_dev(bad))
    assert M.check_perm(_dev(M.random_perm(n, seed=1)))


def test_vector_permute_and_invert(M):
    import torch
    n = 100003
    perm = M.random_perm(n, seed=4)
    x = M.uniform(n, seed=2)
    pd, xd = _dev(perm), _dev(x)
    xp = torch.empty_like(xd)
    M.permute_vector(pd, xd, xp, inverse=False)
    back = torch.empty_like(xd)
    M.permute_vector(pd, xp, back, inverse=True)
    inv = torch.empty_like(pd)
    M.perm_invert(pd, inv)
    torch.cuda.synchronize()
    want = np.empty(n, np.float32)
    want[perm] = x
    assert np.array_equal(xp.cpu().numpy(), want)
    assert np.array_equal(back.cpu().numpy(), x)
    inv_want = np.empty(n, np.int32)
    inv_want[perm] = np.arange(n, dtype=np.int32)
    assert np.array_equal(inv.cpu().numpy(), inv_want)


def test_reorder_merbit_flow_matches_original(M, O, mats):
    """The reference's check (src/class.cu:1435-1445): SpMV on the reordered
    matrix, un-permuted, equals SpMV on the original."""
    import torch
    for name in ("rmat14", "lap48", "heavy"):
        rp, ci, v = mats[name]
        n = rp.size - 1
        p_n2o = M.pgorder(rp, ci, 0, 5)
        perm = np.empty(n, np.int32)
        perm[p_n2o] = np.arange(n, dtype=np.int32)
        pd = _dev(perm)
        A = M.view(_dev(rp), _dev(ci), _dev(v))
        brp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        bci = torch.empty(ci.size, dtype=torch.int32, device="cuda")
        bv = torch.empty(ci.size, dtype=torch.float32, device="cuda")
        M.permute_csr(A, pd, brp, bci, bv)
        B = M.view(brp, bci, bv)
        x = M.uniform(n, seed=31)
        xd = _dev(x)
        xp = torch.empty_like(xd)
        M.permute_vector(pd, xd, xp, inverse=False)
        plan = M.MerbitPlan(B)
        yp = torch.empty_like(xd)
        plan.spmv(xp, yp)
        y = torch.empty_like(xd)
        M.permute_vector(pd, yp, y, inverse=True)
        torch.cuda.synchronize()
        ref = O.spmv_f64(rp, ci, v, x)
        got = y.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-5, name
        plan.close()
