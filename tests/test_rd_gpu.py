"""GPU parity of the reuse-distance features and of the GRAPH-style flow.

Exact RD: integer bin counts must equal the oracle's Fenwick restatement (and
the reference's probabilities from the golden fixtures) exactly.
Sampled RD: sample positions and statuses must equal the oracle's sequential
simulation exactly; estimates must equal the reference kernel's floats bit
for bit when oracle/_ref is built, and the oracle's within 2 ulp (the oracle
uses the host libm's expf/logf).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, csr_random

pytestmark = pytest.mark.gpu

REF_EDGES = [1, 112, 512, 18432, 36864, 73728, 147456, 294912, 589824]
LOG2_EDGES = [1 << k for k in range(0, 13)]


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def streams(M):
    G = np.load(os.path.join(GOLDEN, "golden_host.npz"))
    rng = np.random.default_rng(3)
    out = {name: (G[f"{name}_colidx"], int(G[f"{name}_rowptr"].size - 1)) for name in ("rmat12", "lap24", "band")}
    rp, ci, _ = M.gen_rmat(scale=16, edge_factor=16, seed=1)
    out["rmat16"] = (ci, rp.size - 1)
    out["few_sectors"] = (rng.integers(0, 200, 50000).astype(np.int32), 200)
    out["one_sector"] = (np.full(7000, 5, np.int32), 32)
    out["all_distinct"] = (np.arange(0, 64 * 3000, 32, dtype=np.int32), 64 * 3000)
    out["single"] = (np.array([3], np.int32), 8)
    _, ci, _ = csr_random(20000, 30, seed=4)
    out["random"] = (ci, 20000)
    return out


@pytest.mark.parametrize("name", ["rmat12", "lap24", "band", "rmat16", "few_sectors", "one_sector", "all_distinct",
                                  "single", "random"])
@pytest.mark.parametrize("sector,edges", [(32, REF_EDGES), (32, LOG2_EDGES), (8, REF_EDGES), (1, LOG2_EDGES)])
def test_rd_exact_counts_match_oracle(M, O, streams, name, sector, edges):
    s, ncols = streams[name]
    got, gv = M.rd_hist_exact(_dev(s), ncols, sector, edges)
    want, wv = O.rd_hist_exact(s, ncols, sector, edges)
    assert gv == wv
    assert np.array_equal(got, want)


def test_rd_exact_matches_reference_fixtures(M):
    G = np.load(os.path.join(GOLDEN, "golden_host.npz"))
    for name in ("rmat12", "lap24", "band"):
        ci = G[f"{name}_colidx"]
        n = G[f"{name}_rowptr"].size - 1
        for key, sector, edges in (("rd_ref", 32, REF_EDGES), ("rd_log2", 32, LOG2_EDGES), ("rd_s8", 8, REF_EDGES)):
            c, v = M.rd_hist_exact(_dev(ci), n, sector, edges)
            assert np.array_equal(c / v, G[f"{name}_{key}"]), (name, key)


def test_rd_exact_empty(M):
    import torch
    c, v = M.rd_hist_exact(torch.empty(0, dtype=torch.int32, device="cuda"), 10)
    assert v == 0 and not c.any()


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


@pytest.mark.parametrize("name,samples,cap,max_scan,p", [
    ("rmat16", 30960, 589824, 0, 12),
    ("rmat12", 4000, 589824, 0, 12),
    ("lap24", 3000, 589824, 0, 10),
    ("few_sectors", 5000, 0, 0, 4),
    ("random", 5000, 589824, 3000, 14),
    ("band", 2000, 600000, 100, 12),
])
def test_hll_sampled_matches_oracle(M, O, streams, name, samples, cap, max_scan, p):
    import torch
    s, ncols = streams[name]
    seed = M.hll_seed(7, 0)
    est = torch.empty(samples, dtype=torch.float32, device="cuda")
    st = torch.empty(samples, dtype=torch.int32, device="cuda")
    pos = torch.empty(samples, dtype=torch.int32, device="cuda")
    counts, stats = M.rd_hist_sampled(_dev(s), samples=samples, rd_cap=cap, hll_p=p, max_scan=max_scan, seed=seed,
                                      est=est, status=st, pos=pos)
    oe, ost, opos = O.hll_sampled(s, samples, 32, seed, cap, max_scan, p)
    assert np.array_equal(pos.cpu().numpy(), opos)
    assert np.array_equal(st.cpu().numpy(), ost)
    assert _ulps(est.cpu().numpy(), oe).max() <= 2
    oc, ostats = O.hll_bin(est.cpu().numpy(), st.cpu().numpy())
    assert np.array_equal(counts, oc) and np.array_equal(stats, ostats)


def test_hll_matches_reference_kernel(M, O, streams):
    R = O.ref()
    if R is None:
        pytest.skip("reference build (oracle/_ref) not present")
    import torch
    for name, samples, p in (("rmat16", 30960, 12), ("lap24", 3000, 10), ("few_sectors", 4000, 4)):
        s, _ = streams[name]
        seed = M.hll_seed(3, 1)
        sd = _dev(s)
        est = torch.empty(samples, dtype=torch.float32, device="cuda")
        st = torch.empty(samples, dtype=torch.int32, device="cuda")
        pos = torch.empty(samples, dtype=torch.int32, device="cuda")
        M.rd_hist_sampled(sd, samples=samples, hll_p=p, seed=seed, est=est, status=st, pos=pos)
        rest = torch.empty_like(est)
        rst = torch.empty_like(st)
        rpos = torch.empty_like(pos)
        assert R.ref_hll_sampled(sd.data_ptr(), s.size, samples, 32, seed, 589824, 0, p, rest.data_ptr(),
                                 rst.data_ptr(), rpos.data_ptr()) == 0
        assert torch.equal(pos, rpos), name
        assert torch.equal(st, rst), name
        assert torch.equal(est.view(torch.int32), rest.view(torch.int32)), name


def test_hll_argument_rules(M, streams):
    s, _ = streams["rmat12"]
    sd = _dev(s)
    with pytest.raises(M.MRError):
        M.rd_hist_sampled(sd, samples=10, rd_cap=1000)  # cap below the last edge
    with pytest.raises(M.MRError):
        M.rd_hist_sampled(sd, samples=10, sector=0)
    c, st = M.rd_hist_sampled(sd, samples=0)
    assert not c.any() and not st.any()
    c, st = M.rd_hist_sampled(_dev(np.array([1], np.int32)), samples=10)
    assert not c.any() and not st.any()


def test_locality_predict_matches_oracle_pipeline(M, O, streams):
    s, ncols = streams["rmat16"]
    speedup, feats = M.locality_predict(_dev(s), ncols, graph_id=5)
    oe, ost, _ = O.hll_sampled(s, 30960, 32, M.hll_seed(5, 0), 589824, 0, 12)
    oc, ostats = O.hll_bin(oe, ost)
    valid = ostats[0] + ostats[2]
    of = oc / valid
    assert np.abs(feats - of).max() <= 2.0 / valid  # an estimate within 2 ulp of an edge may bin differently
    assert abs(speedup - M.predict_speedup(feats)) <= 1e-6 * speedup


def test_graph_flow_matches_reference(M, O):
    """GRAPH-style object: gorder4 permutation, then merbit/csr SpMV in the
    original numbering, against the FP64 oracle and (when built) the
    reference's whole gorder4 run on the device."""
    rp, ci, v = M.gen_rmat(scale=14, edge_factor=16, seed=6)
    n = rp.size - 1
    g = M.Graph(rp, ci, v, graph_id=2)
    ms_order, ms_relabel = g.gorder4(vsize=0, width=5)
    perm = g.perm()
    p_n2o = M.pgorder(rp, ci, 0, 5)
    want = np.empty(n, np.int32)
    want[p_n2o] = np.arange(n, dtype=np.int32)
    assert np.array_equal(perm, want)
    x = M.uniform(n, seed=4)
    ref = O.spmv_f64(rp, ci, v, x)
    for method in ("merbit", "csr"):
        y, ms_plan, ms_spmv = g.spmv(method, iters=3, x=x)
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= 1e-5, method
        assert ms_spmv > 0
    y1, _, _ = g.spmv("merbit", iters=1)  # x = 1, as the reference
    assert np.linalg.norm(y1 - O.spmv_f64(rp, ci, v, np.ones(n, np.float32))) <= 1e-5 * np.linalg.norm(y1)
    sp, feats = g.locality_predict()
    assert sp > 0 and abs(feats.sum() - 1.0) < 1e-9
    R = O.ref()
    if R is not None:
        rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
        row_ind, col_ind, vals = _dev(ci.copy()), _dev(rows), _dev(v.copy())
        rperm = np.empty(n, np.int32)
        assert R.ref_gorder4_full(n, int(ci.size), row_ind.data_ptr(), col_ind.data_ptr(), vals.data_ptr(),
                                  M.pgorder_width(n, ci.size), 5, rperm.ctypes.data) == 0
        assert np.array_equal(rperm, perm)
    g.close()
