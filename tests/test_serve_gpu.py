"""Serving loop: continuous batching over a device-resident pool.

Each result must match the FP64 oracle of the stored values (within the
FP32-accumulation tolerance), be bitwise identical alone and in a mixed
batch, survive LRU eviction under a tight HBM budget, and report
admission refusals, timeouts and latency statistics."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pool(M):
    mats = []
    specs = [("rmat", 12, 16), ("band", 20000, 17), ("rmat", 14, 8), ("band", 3000, 3), ("rmat", 13, 24)]
    for i, (kind, a, b) in enumerate(specs):
        if kind == "rmat":
            rp, ci, v = M.gen_rmat(scale=a, edge_factor=b, seed=i + 1)
        else:
            rp, ci, v = M.gen_banded(a, b, seed=i + 1)
        n2o = M.pgorder(rp, ci, 0, 5)
        perm = np.empty(rp.size - 1, np.int32)
        perm[n2o] = np.arange(rp.size - 1, dtype=np.int32)
        # the pool holds the reordered matrix and its permutation
        import pyoracle as O
        brp, bci, bv = O.permute_csr(rp, ci, v, perm)
        mats.append(dict(orig=(rp, ci, v), reordered=(brp, bci, bv), perm=perm))
    return mats


@pytest.fixture(scope="module")
def pool(M):
    return _pool(M)


def _rel(a, b):
    return np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b)


@pytest.mark.parametrize("dtype", [np.float32, np.float16])
def test_results_match_fp64_and_are_identical_alone_and_mixed(M, O, pool, dtype):
    srv = M.Server(window_us=300, max_batch=64, lanes=3)
    ids = []
    for m in pool:
        brp, bci, bv = m["reordered"]
        ids.append(srv.add_matrix(brp, bci, bv.astype(dtype), m["perm"]))
    rng = np.random.default_rng(0)
    reqs = []
    for k in range(24):
        j = int(rng.integers(0, len(pool)))
        n = pool[j]["perm"].size
        reqs.append((j, M.uniform(n, seed=100 + k)))
    # alone: one request at a time
    alone = []
    for j, x in reqs:
        y = np.full(x.size, np.nan, np.float32)
        rc, lat = srv.wait(srv.submit(ids[j], x, y))
        assert rc == M.MR_OK and lat > 0
        alone.append(y)
    # mixed: all at once, batched together
    ys = [np.full(x.size, np.nan, np.float32) for _, x in reqs]
    tickets = [srv.submit(ids[j], x, y) for (j, x), y in zip(reqs, ys)]
    for t in tickets:
        assert srv.wait(t)[0] == M.MR_OK
    for (j, x), ya, ym in zip(reqs, alone, ys):
        assert np.array_equal(ya.view(np.int32), ym.view(np.int32))
        rp, ci, v = pool[j]["orig"]
        vr = v.astype(dtype).astype(np.float32)
        assert _rel(ym, O.spmv_f64(rp, ci, vr, x)) <= 1e-5
    st = srv.stats()
    assert st["completed"] == 48 and st["batches"] < 48 and st["p99_us"] >= st["p50_us"] > 0
    srv.close()


@pytest.mark.parametrize("hub_cache", [False, True])
def test_lru_eviction_under_tight_budget(M, O, pool, hub_cache):
    # resident bytes per matrix: CSR + perm and inverse (+ with the hub cache
    # the remapped colidx and the plan's tables, under 2 MB here)
    sizes = [m["reordered"][1].size * (12 if hub_cache else 8) + m["perm"].size * 16 + (2 << 20 if hub_cache else 0)
             for m in pool]
    srv = M.Server(hbm_budget_bytes=int(sum(sorted(sizes)[-2:]) * 1.3), window_us=100, lanes=2, hub_cache=hub_cache)
    ids = [srv.add_matrix(*m["reordered"], m["perm"]) for m in pool]
    # one request at a time, cycling over a pool larger than the budget: with
    # LRU every matrix is evicted before it is used again
    for rnd in range(3):
        for j, m in enumerate(pool):
            x = M.uniform(m["perm"].size, seed=rnd * 10 + j)
            y = np.empty_like(x)
            assert srv.wait(srv.submit(ids[j], x, y))[0] == M.MR_OK
            rp, ci, v = pool[j]["orig"]
            assert _rel(y, O.spmv_f64(rp, ci, v, x)) <= 1e-5
    st = srv.stats()
    assert st["evictions"] > 0 and st["admissions"] > len(pool)
    assert st["resident_bytes"] <= int(sum(sorted(sizes)[-2:]) * 1.3)
    srv.close()


def test_pinned_and_pageable_vectors_give_identical_results(M, pool):
    import torch
    srv = M.Server(window_us=100, lanes=2)
    ids = [srv.add_matrix(*m["reordered"], m["perm"]) for m in pool]
    jobs = []
    for j, m in enumerate(pool):
        n = m["perm"].size
        x = M.uniform(n, seed=40 + j)
        y = np.full(n, np.nan, np.float32)
        xp = torch.from_numpy(x).pin_memory()
        yp = torch.full((n,), float("nan")).pin_memory()
        jobs.append((srv.submit(ids[j], x, y), srv.submit(ids[j], xp.numpy(), yp.numpy()), y, yp, xp))
    for t_pageable, t_pinned, y, yp, _ in jobs:
        assert srv.wait(t_pageable)[0] == M.MR_OK and srv.wait(t_pinned)[0] == M.MR_OK
        assert np.array_equal(y.view(np.int32), yp.numpy().view(np.int32))
    srv.close()


def test_plain_requests_match_server(M, pool):
    import torch
    plans, views, perms, keep = [], [], [], []
    for m in pool:
        brp, bci, bv = (torch.from_numpy(a).cuda() for a in m["reordered"])
        A = M.view(brp, bci, bv)
        plans.append(M.MerbitPlan(A))
        views.append(A)
        perms.append(torch.from_numpy(m["perm"]).cuda())
    req = np.array([0, 3, 1, 1, 4, 2], np.int32)
    xs = [M.uniform(pool[k]["perm"].size, seed=70 + i) for i, k in enumerate(req)]
    ys = [np.full(x.size, np.nan, np.float32) for x in xs]
    ms, lat = M.plain_requests(plans, views, perms, req, xs, ys)
    assert ms > 0 and lat.size == req.size and (lat > 0).all()
    srv = M.Server(window_us=100)
    ids = [srv.add_matrix(*m["reordered"], m["perm"]) for m in pool]
    for k, x, y in zip(req, xs, ys):
        ys2 = np.empty_like(x)
        assert srv.wait(srv.submit(ids[k], x, ys2))[0] == M.MR_OK
        # same SpMV (FP32 values, sigma 14) up to the plan's block and hub
        # cache, which change the summation order only within FP32 rounding
        assert _rel(ys2, y.astype(np.float64)) <= 1e-6
    srv.close()


def test_refusal_and_timeout(M, pool):
    srv = M.Server(hbm_budget_bytes=1 << 12, window_us=100)
    mid = srv.add_matrix(*pool[0]["reordered"], pool[0]["perm"])
    x = M.uniform(pool[0]["perm"].size, seed=1)
    y = np.empty_like(x)
    rc, _ = srv.wait(srv.submit(mid, x, y))
    assert rc == M.MR_ERR_BUSY  # can never fit the budget
    srv.close()
    slow = M.Server(window_us=2_000_000)
    mid = slow.add_matrix(*pool[3]["reordered"], pool[3]["perm"])
    x = M.uniform(pool[3]["perm"].size, seed=2)
    y = np.empty_like(x)
    t = slow.submit(mid, x, y)
    assert slow.wait(t, timeout_ms=10)[0] == M.MR_ERR_TIMEOUT
    assert slow.wait(t, timeout_ms=10000)[0] == M.MR_OK
    slow.close()
    with pytest.raises(M.MRError):
        M.Server().submit(99, x, y)


def test_loadgen_poisson(M, pool):
    srv = M.Server(window_us=200, lanes=3)
    ids = [srv.add_matrix(*m["reordered"], m["perm"]) for m in pool]
    xs = [M.uniform(m["perm"].size, seed=j) for j, m in enumerate(pool)]
    ys = [np.empty_like(x) for x in xs]
    srv.loadgen(ids, xs, ys, n_requests=2000, rate=5000.0, seed=3)
    st = srv.stats()
    assert st["completed"] == 2000 and st["req_per_s"] > 1000 and st["mean_batch"] >= 1
    # stage timers of every batch: device copies and kernels, host launch work
    assert st["h2d_ms"] > 0 and st["compute_ms"] > 0 and st["d2h_ms"] > 0 and st["launch_ms"] > 0
    srv.reset_stats()
    st = srv.stats()
    assert st["h2d_ms"] == 0 and st["compute_ms"] == 0 and st["launch_ms"] == 0
    srv.close()


def _big_pool(M):
    """Matrices whose vectors straddle the staging threshold (1 MB = 262,144
    floats): R-MAT scale 12 and 15 (staged) and 19 (copied directly when the
    vectors are page-locked)."""
    import pyoracle as O
    mats = []
    for i, sc in enumerate((12, 19, 15)):
        rp, ci, v = M.gen_rmat(scale=sc, edge_factor=8 if sc > 16 else 12, seed=30 + i)
        n2o = M.pgorder(rp, ci, 0, 5)
        perm = np.empty(rp.size - 1, np.int32)
        perm[n2o] = np.arange(rp.size - 1, dtype=np.int32)
        mats.append(dict(orig=(rp, ci, v), reordered=O.permute_csr(rp, ci, v, perm), perm=perm))
    return mats


@pytest.mark.parametrize("hub_cache", [False, True])
def test_staged_and_direct_copies_in_one_batch(M, O, hub_cache):
    """Page-locked vectors above the staging threshold go by their own DMA,
    smaller ones through the staging buffer, in one batch: each result is
    bitwise the one the request gets alone, and within 1e-5 of FP64. With
    the hub cache each matrix runs its own persistent plan."""
    import torch
    mats = _big_pool(M)
    srv = M.Server(window_us=2000, max_batch=16, lanes=2, sigma=20, hub_cache=hub_cache)
    ids = [srv.add_matrix(*m["reordered"], m["perm"]) for m in mats]
    jobs = []
    for k in range(9):
        j = k % 3
        n = mats[j]["perm"].size
        x = torch.from_numpy(M.uniform(n, seed=200 + k)).pin_memory()
        y = torch.full((n,), float("nan")).pin_memory()
        jobs.append((j, x, y))
    alone = []
    for j, x, y in jobs:
        ya = np.full(x.numel(), np.nan, np.float32)
        assert srv.wait(srv.submit(ids[j], x.numpy(), ya))[0] == M.MR_OK
        alone.append(ya)
    tickets = [srv.submit(ids[j], x.numpy(), y.numpy()) for j, x, y in jobs]
    for t in tickets:
        assert srv.wait(t)[0] == M.MR_OK
    assert srv.stats()["batches"] < 9 + 9  # the burst was batched
    for (j, x, y), ya in zip(jobs, alone):
        assert np.array_equal(ya.view(np.int32), y.numpy().view(np.int32))
        rp, ci, v = mats[j]["orig"]
        assert _rel(y.numpy(), O.spmv_f64(rp, ci, v, x.numpy())) <= 1e-5
    srv.close()


@pytest.mark.parametrize("dtype", [np.float32, np.float16, "bf16"])
def test_hub_cache_server_matches_batched_server(M, pool, dtype):
    """The same requests through a server of batched plans and one of
    persistent hub-cache plans, for FP32, FP16 and BF16 values: the same SpMV
    up to summation order."""
    import torch
    outs = []
    for hub in (False, True):
        srv = M.Server(window_us=200, lanes=3, hub_cache=hub)
        ids = []
        for m in pool:
            brp, bci, bv = m["reordered"]
            if dtype == "bf16":
                vals = torch.from_numpy(bv).to(torch.bfloat16)
            else:
                vals = bv.astype(dtype)
            ids.append(srv.add_matrix(brp, bci, vals, m["perm"]))
        ys = []
        for j, m in enumerate(pool):
            x = M.uniform(m["perm"].size, seed=300 + j)
            y = np.full(x.size, np.nan, np.float32)
            assert srv.wait(srv.submit(ids[j], x, y))[0] == M.MR_OK
            ys.append(y)
        srv.close()
        outs.append(ys)
    for a, b in zip(*outs):
        assert _rel(b, a.astype(np.float64)) <= 1e-6
