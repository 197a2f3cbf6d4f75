"""Comparator permutation producers on the GPU (degree, DBG, random): the
degree and DBG orders equal the oracle's restatement of GRAPH::relabel_degree
/ GRAPH::dbg and the reference's own functions run on the B200; the random
order equals the oracle's restatement of GRAPH::relabel_random and the
reference's own relabel_random (thrust::shuffle) run on the B200."""
import numpy as np
import pytest

from conftest import csr_random

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def mats(M):
    return {
        "rmat14": M.gen_rmat(scale=14, edge_factor=16, seed=2),
        "chung_lu": M.gen_chung_lu(1 << 15, 2.1, 20.0, 1, 3000, seed=4),
        "lap64": M.gen_laplace2d(64, shuffle=True, seed=1),
        "random": csr_random(5000, 70, seed=8, empty_frac=0.3),
        "band": M.gen_banded(3000, 9, seed=2),
    }


def _run(M, fn, rp, ci, v):
    import torch
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    p = torch.empty(rp.size - 1, dtype=torch.int32, device="cuda")
    fn(A, p)
    torch.cuda.synchronize()
    return p.cpu().numpy()


@pytest.mark.parametrize("name", ["rmat14", "chung_lu", "lap64", "random", "band"])
def test_degree_and_dbg_match_oracle(M, O, mats, name):
    rp, ci, v = mats[name]
    assert np.array_equal(_run(M, M.order_degree, rp, ci, v), O.order_degree(rp, ci))
    assert np.array_equal(_run(M, M.order_dbg, rp, ci, v), O.order_dbg(rp, ci))


@pytest.mark.parametrize("kind", [0, 1])
def test_degree_and_dbg_match_reference(M, O, mats, kind):
    R = O.ref()
    if R is None:
        pytest.skip("reference build (oracle/_ref) not present")
    fn = M.order_degree if kind == 0 else M.order_dbg
    for name in ("rmat14", "chung_lu", "random"):
        rp, ci, v = mats[name]
        n = rp.size - 1
        rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
        row_ind, col_ind, vals = _dev(ci.copy()), _dev(rows), _dev(v.copy())  # reference layout
        ref = np.empty(n, np.int32)
        assert R.ref_relabel_order(kind, n, int(ci.size), row_ind.data_ptr(), col_ind.data_ptr(), vals.data_ptr(), 7,
                                   ref.ctypes.data) == 0
        assert np.array_equal(_run(M, fn, rp, ci, v), ref), name


def test_random_order_is_a_seeded_bijection(M):
    import torch
    n = 100003
    a = torch.empty(n, dtype=torch.int32, device="cuda")
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    M.order_random(n, 5, a)
    M.order_random(n, 5, b)
    M.order_random(n, 6, c)
    torch.cuda.synchronize()
    pa = a.cpu().numpy()
    assert np.array_equal(np.sort(pa), np.arange(n))
    assert torch.equal(a, b) and not torch.equal(a, c)
    # no long identity runs: a shuffle, not a near-identity map
    assert np.mean(pa == np.arange(n)) < 1e-3
    assert M.check_perm(a)


@pytest.mark.parametrize("n", [1, 16, 17, 4096, 100003, 1 << 20, 4194304])
def test_random_order_matches_oracle(M, O, n):
    import torch
    for seed in (0, 1, 7):
        p = torch.empty(n, dtype=torch.int32, device="cuda")
        M.order_random(n, seed, p)
        torch.cuda.synchronize()
        assert np.array_equal(p.cpu().numpy(), O.order_random(n, seed)), (n, seed)


def test_random_order_matches_reference_relabel_random(M, O, mats):
    """GRAPH::relabel_random itself (thrust::shuffle on the device, seeded
    with graph_id) on the B200: the same permutation and, applied through
    mr_permute_csr, the same relabelled matrix."""
    R = O.ref()
    if R is None:
        pytest.skip("reference build (oracle/_ref) not present")
    import torch
    for name, gid in (("rmat14", 0), ("chung_lu", 7), ("random", 123)):
        rp, ci, v = mats[name]
        n = rp.size - 1
        rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
        row_ind, col_ind, vals = _dev(ci.copy()), _dev(rows), _dev(v.copy())  # reference layout
        ref = np.empty(n, np.int32)
        assert R.ref_relabel_order(2, n, int(ci.size), row_ind.data_ptr(), col_ind.data_ptr(), vals.data_ptr(), gid,
                                   ref.ctypes.data) == 0
        p = torch.empty(n, dtype=torch.int32, device="cuda")
        M.order_random(n, gid, p)
        A = M.view(_dev(rp), _dev(ci), _dev(v))
        orp = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        oci = torch.empty(ci.size, dtype=torch.int32, device="cuda")
        ov = torch.empty(ci.size, dtype=torch.float32, device="cuda")
        M.permute_csr(A, p, orp, oci, ov)
        torch.cuda.synchronize()
        assert np.array_equal(p.cpu().numpy(), ref), name
        g_rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(orp.cpu().numpy()))
        assert np.array_equal(col_ind.cpu().numpy(), g_rows), name
        assert np.array_equal(row_ind.cpu().numpy(), oci.cpu().numpy()), name
        assert np.array_equal(vals.cpu().numpy().view(np.uint32), ov.cpu().numpy().view(np.uint32)), name


def test_invalid_input_rejected(M):
    import torch
    rp = np.array([0, 2, 3], np.int32)
    ci = np.array([0, 5, 1], np.int32)  # column 5 out of range for n = 2
    A = M.view(_dev(rp), _dev(ci), _dev(np.ones(3, np.float32)))
    p = torch.empty(2, dtype=torch.int32, device="cuda")
    with pytest.raises(M.MRError):
        M.order_degree(A, p)
