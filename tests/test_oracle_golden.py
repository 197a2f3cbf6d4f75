"""Pins the CPU oracle and the product's host code to the reference.

Fixtures in tests/golden/golden_host.npz come from the reference's own code,
those in golden_random.npz from Thrust's shuffle that the reference's
relabel_random calls (tests/golden/make_golden.py). When oracle/_ref is built
in this container the same functions are also compared live on larger inputs.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

G = np.load(os.path.join(GOLDEN, "golden_host.npz"))
CASES = ["rmat12", "lap24", "band"]
LOG2_EDGES = [1 << k for k in range(0, 13)]
REF_EDGES = [1, 112, 512, 18432, 36864, 73728, 147456, 294912, 589824]


def _probs(counts, valid):
    return counts / valid if valid else np.zeros(counts.size)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("key,vs,w", [("v1024_w5", 1024, 5), ("v256_w5", 256, 5), ("v64_w5", 64, 5),
                                      ("v256_w1", 256, 1)])
def test_pgorder_oracle_and_product_match_reference(O, M, case, key, vs, w):
    rp, ci = G[f"{case}_rowptr"], G[f"{case}_colidx"]
    want = G[f"{case}_perm_{key}"]
    assert np.array_equal(O.pgorder(rp, ci, vs, w), want)
    assert np.array_equal(M.pgorder(rp, ci, vs, w, threads=3), want)


@pytest.mark.parametrize("case", CASES)
def test_rd_exact_oracle_matches_reference(O, case):
    rp, ci = G[f"{case}_rowptr"], G[f"{case}_colidx"]
    n = rp.size - 1
    c, v = O.rd_hist_exact(ci, n, 32, REF_EDGES)
    assert np.array_equal(_probs(c, v), G[f"{case}_rd_ref"])
    c, v = O.rd_hist_exact(ci, n, 32, LOG2_EDGES)
    assert np.array_equal(_probs(c, v), G[f"{case}_rd_log2"])
    c, v = O.rd_hist_exact(ci, n, 8, REF_EDGES)
    assert np.array_equal(_probs(c, v), G[f"{case}_rd_s8"])


def test_width_oracle_and_product_match_reference(O, M):
    for (n, nnz), want in zip(G["width_sizes"], G["width_ref"]):
        assert O.get_width(int(n), int(nnz)) == want
        assert M.pgorder_width(int(n), int(nnz)) == want


def test_predictor_matches_reference(M):
    for f, want in zip(G["predict_features"], G["predict_ref"]):
        assert M.predict_speedup(f, M.MODEL_MERBIT_SAMPLED) == want


def test_predictor_rejects_nonfinite(M):
    with pytest.raises(M.MRError) as e:
        M.predict_speedup([1e300] * 10, M.MODEL_MERBIT_SAMPLED)
    assert e.value.code == M.MR_ERR_PREDICT


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "libmr_ref.so")),
                    reason="reference build (oracle/_ref) not present")
class TestLiveReference:
    """Larger seeded inputs against the reference compiled from its sources."""

    def test_pgorder_rmat16(self, O, M):
        rp, ci, _ = M.gen_rmat(scale=16, edge_factor=16, seed=1)
        want = O.ref_pgorder(rp, ci, 1024, 5)
        assert np.array_equal(M.pgorder(rp, ci, 0, 5), want)
        assert np.array_equal(O.pgorder(rp, ci, 1024, 5), want)

    def test_pgorder_laplace_vsize16384(self, O, M):
        rp, ci, _ = M.gen_laplace2d(160, shuffle=True, seed=9)
        n = rp.size - 1
        assert M.pgorder_width(n, ci.size) == O.ref_get_width(n, ci.size)
        want = O.ref_pgorder(rp, ci, 16384, 5)
        assert np.array_equal(M.pgorder(rp, ci, 16384, 5), want)

    def test_rd_exact_rmat16(self, O, M):
        rp, ci, _ = M.gen_rmat(scale=16, edge_factor=16, seed=1)
        n = rp.size - 1
        c, v = O.rd_hist_exact(ci, n, 32, REF_EDGES)
        assert np.array_equal(_probs(c, v), O.ref_rd_probs(ci, n, 32, REF_EDGES))

    def test_predictor_models_follow_reference_formula(self, O, M):
        rng = np.random.default_rng(5)
        for _ in range(20):
            f = rng.dirichlet(np.ones(10))
            assert M.predict_speedup(f) == O.ref_predict(f)


R_FIX = np.load(os.path.join(GOLDEN, "golden_random.npz"))


@pytest.mark.parametrize("n,seed", [tuple(int(a) for a in c) for c in R_FIX["cases"]])
def test_random_order_oracle_matches_thrust_shuffle(O, n, seed):
    """GRAPH::relabel_random's permutation (thrust::shuffle, seeded with
    graph_id): the oracle's restatement against fixtures from Thrust's own
    implementation (tests/golden/make_golden.py)."""
    got = O.order_random(n, seed)
    assert np.array_equal(got, R_FIX[f"perm_{n}_{seed}"])
    assert np.array_equal(np.sort(got), np.arange(n))


def test_random_order_oracle_matches_thrust_live(O):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    for n, seed in ((100003, 0), (1 << 20, 12345), (3, 9)):
        assert np.array_equal(O.order_random(n, seed), O.ref_shuffle(n, seed)), (n, seed)
