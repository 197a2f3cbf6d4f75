"""The bench line's bookkeeping, on the CPU: the roofline's DRAM traffic is
read from the committed ncu summary of exactly the headline plan (R-MAT s22,
SIGMA 14, 1024 threads, hub cache), and both arms print one workload
config."""
import argparse
import os

import bench


def _args(**kw):
    a = argparse.Namespace(scale=22, edge_factor=16, seed=1)
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def test_traffic_comes_from_the_capture_of_the_headline_plan():
    name = "merbit_persistent_hub_rmat_s22_sigma14.md"
    assert os.path.exists(os.path.join(bench.REPO, "profiles", name))
    b = bench.spmv_bytes(4194304, 65244768)
    assert b == 572289796
    traffic, src = bench.traffic_from_profiles(name, b)
    assert src == name and traffic == 576536320
    # scaled by algorithmic bytes for another size of the same family
    t2, _ = bench.traffic_from_profiles(name, b // 2)
    assert abs(t2 - 576536320 / 2) <= 1


def test_missing_capture_gives_no_traffic():
    assert bench.traffic_from_profiles("no_such_capture.md", 1000) == (None, None)


def test_both_arms_share_the_workload_config():
    a = _args()
    ours = bench.workload_config(a, 4194304, 65244768)
    assert ours == {"workload": "rmat_s22_ef16 pGOrder-reordered FP32 SpMV", "n_rows": 4194304,
                    "nnz": 65244768, "seed": 1}
    assert "MERBIT" not in ours["workload"] and "CSR" not in ours["workload"]


def test_headline_runs_a_fixed_plan_by_default():
    a = bench.parser().parse_args([])
    assert (a.tune, a.sigma, a.block, a.gpus, a.impl) == (False, 14, 1024, 1, "ours")
    assert bench.parser().parse_args(["--tune"]).tune
    assert not bench.parser().parse_args(["--no-tune"]).tune
    # the e2e leg has its own request count, independent of --steps
    assert bench.parser().parse_args(["--steps", "20"]).e2e_steps == 400
