"""Generates the host-side golden fixtures from the reference's own code.

Runs the reference functions compiled from its sources (oracle/_ref, built by
oracle/build_ref.sh from the reference checkout) on small seeded inputs and
stores inputs and outputs in tests/golden/golden_host.npz:

  * pGOrder permutations (order_on_cpu driven as GRAPH::gorder4 does,
    src/class.cu:2647-2683),
  * exact RD bin probabilities (compute_sector_rd_histogram,
    src/class.cu:892-936) for the reference bins and log2 bins,
  * GRAPH::get_width over a grid of sizes (src/class.cu:733-750),
  * rd_merbit_model::PredictSpeedup on feature vectors (include/model.cuh),
  * the band gate's decision counts (run_band_gate_scan,
    ridge/train.py:983-1026, imported from the reference checkout named by
    MR_REFERENCE, default the `reference` directory beside this
    repository) on seeded predicted / true
    speedups for every BAND_GATE_PAIRS entry.

Usage: python tests/golden/make_golden.py   (needs oracle/_ref built)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "matrix-reorder_b200"))

import mrb200 as M  # noqa: E402  (generators only)
import pyoracle as O  # noqa: E402

LOG2_EDGES = [1 << k for k in range(0, 13)]


RANDOM_CASES = [(1, 0), (16, 3), (17, 1), (1000, 0), (4096, 42), (30011, 7)]


def random_orders() -> None:
    """tests/golden/golden_random.npz: the permutation GRAPH::relabel_random
    draws (src/class.cu:1467-1473), from Thrust's own shuffle run through the
    reference build's host entry point, for (n, graph_id) pairs."""
    assert O.ref_available(), "build oracle/_ref first (oracle/build_ref.sh)"
    out = {"cases": np.array(RANDOM_CASES, np.int64)}
    for n, seed in RANDOM_CASES:
        out[f"perm_{n}_{seed}"] = O.ref_shuffle(n, seed)
    np.savez_compressed(os.path.join(HERE, "golden_random.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_random.npz"))


def main() -> None:
    assert O.ref_available(), "build oracle/_ref first (oracle/build_ref.sh)"
    random_orders()
    out = {}
    cases = {
        "rmat12": M.gen_rmat(scale=12, edge_factor=8, seed=3)[:2],
        "lap24": M.gen_laplace2d(24, shuffle=True, seed=5)[:2],
        "band": M.gen_banded(3000, 9, seed=2)[:2],
    }
    for name, (rp, ci) in cases.items():
        n = rp.size - 1
        out[f"{name}_rowptr"] = rp
        out[f"{name}_colidx"] = ci
        for vs in (1024, 256, 64):
            out[f"{name}_perm_v{vs}_w5"] = O.ref_pgorder(rp, ci, vs, 5)
        out[f"{name}_perm_v256_w1"] = O.ref_pgorder(rp, ci, 256, 1)
        out[f"{name}_rd_ref"] = O.ref_rd_probs(ci, n, 32)
        out[f"{name}_rd_log2"] = O.ref_rd_probs(ci, n, 32, LOG2_EDGES)
        out[f"{name}_rd_s8"] = O.ref_rd_probs(ci, n, 8)
    sizes = []
    for n in (1000, 4096, 65536, 1 << 20, 4194304, 8388608, 16777216):
        for deg in (1, 2, 3, 4, 5, 8, 16, 20, 64, 200):
            if n * deg < 2**31:  # the reference takes int sizes
                sizes.append((n, n * deg))
    sizes.append((100, 50))  # nnz / n == 0
    sizes = np.array(sizes, np.int64)
    out["width_sizes"] = sizes
    out["width_ref"] = np.array([O.ref_get_width(int(a), int(b)) for a, b in sizes], np.int32)
    rng = np.random.default_rng(11)
    feats = rng.dirichlet(np.ones(10), size=16)
    out["predict_features"] = feats
    out["predict_ref"] = np.array([O.ref_predict(f) for f in feats])
    # band gate of the ridge trainer, run by the reference's own Python
    # the reference checkout sits beside this repository unless MR_REFERENCE names it
    ref = os.environ.get("MR_REFERENCE", os.path.join(os.path.dirname(REPO), "reference"))
    sys.path.insert(0, os.path.join(ref, "ridge"))
    import pandas as pd
    import train as T  # the reference's ridge/train.py
    pred = np.concatenate([rng.lognormal(0.0, 0.05, 400),
                           np.array([t for pair in T.BAND_GATE_PAIRS for t in pair])])  # exactly on the thresholds
    true = rng.lognormal(0.0, 0.08, pred.size)
    scan = T.run_band_gate_scan(pd.DataFrame({"speedup": true, "pred_speedup": pred}), T.BAND_GATE_PAIRS)
    out["gate_pred"] = pred
    out["gate_true"] = true
    out["gate_pairs"] = np.array(T.BAND_GATE_PAIRS, np.float64)
    out["gate_counts"] = scan[["tp", "tn", "fp", "fn", "num_decided"]].to_numpy(np.int64)
    np.savez_compressed(os.path.join(HERE, "golden_host.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_host.npz"))


if __name__ == "__main__":
    main()
