"""Predictor-gated reorder. CPU: the band gate's decisions reproduce the
decision counts of the reference trainer's run_band_gate_scan
(ridge/train.py:983-1026) for every scanned (tau_l, tau_h) pair, on the
golden fixtures generated from the reference's own Python. GPU: the exact-RD
features equal the oracle's histogram, the predicted value is the ridge
model of those features, and the gated pipeline reorders exactly when the
gate says so."""
import os

import numpy as np
import pytest

from conftest import REPO

G = np.load(os.path.join(REPO, "tests", "golden", "golden_host.npz"))


def test_band_gate_matches_reference_scan(M):
    pred, true = G["gate_pred"], G["gate_true"]
    for (tl, th), want in zip(G["gate_pairs"], G["gate_counts"]):
        d = np.array([M.band_gate(float(p), float(tl), float(th)) for p in pred])
        decided = d != M.GATE_UNCERTAIN
        pos = d[decided] == M.GATE_RELABEL
        act = true[decided] > 1.0
        got = [np.sum(pos & act), np.sum(~pos & ~act), np.sum(pos & ~act), np.sum(~pos & act), decided.sum()]
        assert got == list(want), (tl, th)


def test_band_gate_edges(M):
    assert M.band_gate(1.05, 0.95, 1.05) == M.GATE_RELABEL
    assert M.band_gate(0.95, 0.95, 1.05) == M.GATE_SKIP
    assert M.band_gate(1.0, 0.95, 1.05) == M.GATE_UNCERTAIN
    assert M.band_gate(1.0, 1.2, 0.8) == M.GATE_SKIP  # both hold: skip is applied last, as in the trainer
    assert M.band_gate(float("nan"), 0.95, 1.05) == M.GATE_UNCERTAIN
    with pytest.raises(M.MRError):
        M.band_gate(1.0, float("nan"), 1.05)
    assert M.BAND_GATE_PAIRS == [tuple(p) for p in G["gate_pairs"].tolist()]


@pytest.mark.gpu
def test_predict_reorder_exact_and_sampled(M, O):
    import torch
    rp, ci, _ = M.gen_rmat(scale=14, edge_factor=16, seed=5)
    n = rp.size - 1
    s = torch.from_numpy(ci).cuda()
    sp, f = M.predict_reorder(s, n, graph_id=3, model=M.MODEL_MERBIT_EXACT)
    counts, valid = O.rd_hist_exact(ci, n, 32)
    assert np.array_equal(f, counts / valid)
    assert sp == M.predict_speedup(f, M.MODEL_MERBIT_EXACT)
    sp2, f2 = M.predict_reorder(s, n, graph_id=3, model=M.MODEL_MERBIT_SAMPLED)
    sp3, f3 = M.locality_predict(s, n, graph_id=3)
    assert np.array_equal(f2, f3) and np.float32(sp2) == np.float32(sp3)
    sp4, f4 = M.predict_reorder(s, n, graph_id=3, model=M.MODEL_CSR_SAMPLED)
    assert np.array_equal(f4, f2) and sp4 == M.predict_speedup(f2, M.MODEL_CSR_SAMPLED)


@pytest.mark.gpu
def test_gated_reorder_follows_the_gate(M):
    rp, ci, v = M.gen_rmat(scale=13, edge_factor=16, seed=9)
    n = rp.size - 1
    for tl, th, want in ((1e9, 2e9, M.GATE_SKIP), (-1.0, 0.0, M.GATE_RELABEL), (-1.0, 1e9, M.GATE_UNCERTAIN)):
        g = M.Graph(rp, ci, v, graph_id=1)
        d, p = g.gated_reorder(M.MODEL_MERBIT_SAMPLED, tl, th)
        assert d == want and p > 0
        moved = not np.array_equal(g.perm(), np.arange(n, dtype=np.int32))
        assert moved == (d == M.GATE_RELABEL)
        if moved:  # the gated path is gorder4: same permutation as calling it directly
            h = M.Graph(rp, ci, v, graph_id=1)
            h.gorder4(0, 5)
            assert np.array_equal(g.perm(), h.perm())
            h.close()
        y, _, _ = g.spmv("merbit", 1, M.uniform(n, seed=2))
        g.close()
    g = M.Graph(rp, ci, v, graph_id=1)
    d, _ = g.gated_reorder(M.MODEL_MERBIT_SAMPLED, -1.0, 1e9, relabel_uncertain=True)
    assert d == M.GATE_UNCERTAIN and not np.array_equal(g.perm(), np.arange(n, dtype=np.int32))
    g.close()
